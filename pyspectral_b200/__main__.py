import sys

from pyspectral_b200.cli import main

sys.exit(main())
