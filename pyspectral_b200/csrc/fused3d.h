// Host launchers of the fused 3D engine (kernels in fused3d.cuh, compiled in fused3d.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace sp {
namespace fused3 {

// True when the fused 3D engine has kernels for grid n: a power of two, 16..512 (fp32, fp64).
bool supported(int n, int fp64);
// Bytes of the two work arrays, B_spec (n x slots x (2KM+1) x kz) and B_phys
// (n x slots x n x kz); kz padded to whole pairs, slots 5 (Basdevant) / 6 (rotational).
size_t spec_bytes(int n, int fp64, int rot);
size_t phys_bytes(int n, int fp64, int rot);
// Opt the X pass into its dynamic shared memory (once per process and size).
cudaError_t set_attributes(int n, int fp64, int rot);

// Inverse along y of fields f < nfields: B_spec -> B_phys.
cudaError_t y_inverse(int n, int fp64, int rot, const void* Bs, void* Bp, int nfields,
                      const void* tw, cudaStream_t st);
// Forward along y of fields f < nfields, kept ky only: B_phys -> B_spec.
cudaError_t y_forward(int n, int fp64, int rot, const void* Bp, void* Bs, int nfields,
                      const void* tw, cudaStream_t st);
// Z pass in place on B_phys.  mode 0: the stage (inverse, products, forward); mode 1: the
// velocity's max |u_i| only, into umax[0..3) (double bit patterns; atomicMax, zero them first).
// want_max: also record max |u_i| in mode 0.
cudaError_t z_pass(int n, int fp64, int rot, int mode, void* Bp, const void* tw,
                   unsigned long long* umax, int want_max, cudaStream_t st);
// X pass in place on B_spec with the compact state and accumulator; stage -1 builds the
// stage-0 inputs from the state, 0..3 a Lawson stage.
cudaError_t x_pass(int n, int fp64, int rot, int stage, void* Bs, void* u0, void* acc,
                   const void* tab, const void* params, const void* tw, cudaStream_t st);
// Bytes of the compact state (and of the compact accumulator): the kept modes of the three
// components, [c][ky'][kz][kx'].
size_t compact_bytes(int n, int fp64);
// Kept modes of the NumPy-layout state u0 into the compact copy (in != 0) or back.
cudaError_t state_move(int fp64, void* u0, void* compact, int n, int in, cudaStream_t st);
// Zero every mode outside the 2/3 mask of the three state components.
cudaError_t mask(int fp64, void* u0, int n, cudaStream_t st);

}  // namespace fused3
}  // namespace sp
