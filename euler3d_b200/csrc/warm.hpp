// Device helpers around the solver state that are not part of the residual
// path: per-cell features for the warm-start surrogate, writing a predicted
// conservative state into the solver, and widening an FP32 solver to FP64.
#pragma once
#include <cuda_runtime.h>

namespace e3d {

// Per-slot FP64 geometry of the fused path from the per-face arrays: unit
// normal and area (face orientation), area vector signed outward for the
// slot's owner, and the owner's r-vector.  sS may be null.
void launch_slot_geometry64(int NS, const int* slot_face, const int* slot_mate, const double* S, const double* nhat,
                            const double* area, const double* rl, const double* rr, double* sgeo, double* sS,
                            double* srv, cudaStream_t st);

// FP64 copy of an FP32 packed primitive state, into both ping-pong buffers
// (only P0 when P1 is null).
// With W (the carried FP64 conservative state, [5][NR]) the real cells are
// recomputed from it exactly; ghost cells are widened from P32.
void launch_widen_state(int NA, int NR, const float* P32, const double* W, double gm1, double* P0, double* P1,
                        cudaStream_t st);

// FP32 copy of an FP64 packed primitive state (all NA cells)
void launch_narrow_state(int NA, const double* P64, float* P32, cudaStream_t st);

// Raw surrogate inputs of every real cell, [NR][8] floats:
// x, y, z (centroid), distance to the nearest wall-face centre of the cell's
// case, Mach, alpha (degrees), 0, 0.  Cells of a case without wall faces get
// distance 1.
void launch_cell_features(int NR, int nb, const int* roff, const int* block_case, const float* centroid,
                          const int* case_wall_off, const int* wall_face, const double* fc, const float* case_mach_aoa,
                          float* out, cudaStream_t st);

// Writes a conservative state (rho, rho u, rho v, rho w, rho E), [NR][ld]
// floats, into the real cells: primitives of both ping-pong buffers (T) and,
// when W is non-null, the carried FP64 state.  A cell whose prediction is not
// physical (non-finite, rho or p below 1e-3 of freestream) keeps the
// freestream state of its case.  Returns nothing; the count of such cells is
// added to *n_fallback (device int).
template <class T>
void launch_apply_conservative(int NR, int NA, int nb, const int* roff, const int* block_case, const float* Wpred,
                               int ld, const double* case_free, double gamma, T* P0, T* P1, double* W,
                               int* n_fallback, cudaStream_t st);

// Conservative state of every real cell from the packed primitives, [NR][8]
// floats (5 used).
template <class T>
void launch_prims_to_conservative(int NR, int NA, const T* P, double gamma, float* out, cudaStream_t st);

}  // namespace e3d
