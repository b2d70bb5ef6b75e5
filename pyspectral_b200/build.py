"""Build libspectral_b200.so in-tree with nvcc for sm_100a (B200).

``python -m pyspectral_b200.build`` compiles every ``csrc/*.cu`` into one shared library next to
this file.  The library is rebuilt only when a source or header is newer than it (``force=True``
always rebuilds).  nvcc cross-compiles, so this runs on a machine without a GPU.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libspectral_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (set NVCC or put CUDA's bin/ on PATH)")


def _cuda_home(nvcc: str) -> Path:
    return Path(nvcc).resolve().parent.parent


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _deps() -> list[Path]:
    return sources() + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def needs_build(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def _flags(extra: list[str] | None = None) -> list[str]:
    return [*ARCH, "-lineinfo", "-O3", "-std=c++20", "--expt-relaxed-constexpr",
            "-Xcompiler", "-fPIC,-O3,-Wall", f"-I{INCLUDE}", f"-I{CSRC}", *(extra or [])]


def command(out: Path = LIB, extra: list[str] | None = None) -> list[str]:
    """Single nvcc command that compiles every source and links the library."""
    nvcc = _nvcc()
    cuda = _cuda_home(nvcc)
    return [nvcc, *_flags(extra), "-shared", "-o", str(out), *[str(s) for s in sources()],
            f"-L{cuda / 'lib64'}", "-lcufft", f"-Xlinker=-rpath,{cuda / 'lib64'}"]


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compile the library if needed and return its path.  Translation units are compiled in
    parallel (one nvcc per .cu) into a temporary directory, then linked."""
    if not force and not extra and not needs_build():
        return LIB
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    nvcc = _nvcc()
    cuda = _cuda_home(nvcc)
    with tempfile.TemporaryDirectory(prefix="spb200_") as tmpd:
        objs = [Path(tmpd) / (src.stem + ".o") for src in sources()]

        def compile_one(pair: tuple[Path, Path]) -> subprocess.CompletedProcess:
            src, obj = pair
            cmd = [nvcc, *_flags(extra), "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            return subprocess.run(cmd, capture_output=True, text=True)

        with ThreadPoolExecutor(max_workers=max(1, min(len(objs), os.cpu_count() or 1))) as ex:
            results = list(ex.map(compile_one, zip(sources(), objs)))
        for src, res in zip(sources(), results):
            if verbose and (res.stdout or res.stderr):
                print(res.stdout + res.stderr, flush=True)
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src.name} ({res.returncode}):\n"
                                   f"{res.stdout}\n{res.stderr}")
        tmp = LIB.with_suffix(".so.tmp")
        link = [nvcc, *ARCH, "-shared", "-o", str(tmp), *[str(o) for o in objs],
                f"-L{cuda / 'lib64'}", "-lcufft", f"-Xlinker=-rpath,{cuda / 'lib64'}"]
        res = subprocess.run(link, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
        tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    args = sys.argv[1:]
    ptxas = "--ptxas-v" in args
    p = build(force=True, verbose=True, extra=["-Xptxas", "-v"] if ptxas else None)
    print(p)
