/*
 * e3d_oracle.h -- CPU restatement of the euler3D residual/update path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle for the GPU kernels:
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may call it;
 * the euler3d_b200 product never links or calls it.
 *
 * It restates the reference algorithm in the reference's own formulation:
 * face loops that scatter +flux to the left cell and -flux to the right cell
 * (FluxScheme.cpp:100-207), cell loops for gradients and limiters, marker loops
 * for boundary conditions, with the reference's expression order, so an FP64
 * build without contraction (-ffp-contract=off) reproduces the reference bit
 * for bit.  Pinned against arrays dumped by the compiled reference
 * (tests/golden, tests/test_oracle.py).
 *
 * Layouts (one block, block-local ids; real cells first, then ghosts):
 *   prim, limiter      [5][n_all]          conv_res, diss_res, w0   [5][n_all]
 *   grad               [5][n_all][3]       dt, spectral_radius      [n_real]
 *   face_cells [2F], face_normal/face_center/r_left/r_right [3F], face_area [F],
 *   cell_face_ptr [n_all+1], cell_faces/cell_cells [cell_face_ptr[n_all]],
 *   ls_weights [3 * cell_face_ptr[n_real]]
 */
#ifndef E3D_ORACLE_H
#define E3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct e3d_oracle_block {
	int n_real, n_all, n_faces;
	const int* face_cells;
	const double* face_normal;
	const double* face_area;
	const double* face_center;
	const double* r_left;
	const double* r_right;
	const int* cell_face_ptr;
	const int* cell_faces;
	const int* cell_cells;
	const double* cell_volume;
	const double* ls_weights;
	int n_markers, n_real_boundaries;
	const int* marker_kind; /* 1 wall, 2 farfield, 3 symmetry, 4 connexion */
	const int* marker_size;
	const int* marker_cells; /* concatenated ghost ids */
	int n_wall_faces;
	const int* wall_faces;
	/* state (written) */
	double *prim, *conv_res, *diss_res, *w0, *grad, *limiter, *dt, *spectral_radius;
} e3d_oracle_block;

typedef struct e3d_oracle_params {
	double gamma, cfl, mach, aoa_deg, cmac, omega, k;
	int stages, order, flux, gradient, limiter; /* flux 0 roe 1 ausm; gradient 0 GG 1 LS; limiter 0 BJ 1 V */
	int smoothing; /* 1: central implicit residual smoothing in every stage */
} e3d_oracle_params;

/* one inter-block copy list (ConnexionCellIds) */
typedef struct e3d_oracle_connexion {
	int dest_block, origin_block, n;
	const int* dest_cells;
	const int* origin_cells;
} e3d_oracle_connexion;

void e3d_oracle_freestream(const e3d_oracle_params* p, double q[5]);
void e3d_oracle_init_state(e3d_oracle_block* b, const e3d_oracle_params* p);
void e3d_oracle_save_w0(e3d_oracle_block* b, const e3d_oracle_params* p);
void e3d_oracle_spectral_radius(e3d_oracle_block* b, const e3d_oracle_params* p);
void e3d_oracle_timestep(e3d_oracle_block* b, const e3d_oracle_params* p);
void e3d_oracle_gradients(e3d_oracle_block* b, int kind);
void e3d_oracle_limiters(e3d_oracle_block* b, int kind, double omega, double k);
void e3d_oracle_flux_conv(e3d_oracle_block* b, const e3d_oracle_params* p);
void e3d_oracle_flux_diss(e3d_oracle_block* b, const e3d_oracle_params* p, double beta);
void e3d_oracle_update_internal(e3d_oracle_block* b, const e3d_oracle_params* p, double alpha);
void e3d_oracle_update_boundary(e3d_oracle_block* b, const e3d_oracle_params* p);
/* CentralIrsSmoother::smoothResidual; the dissipative v/w start values follow the other eight arrays */
void e3d_oracle_smooth(e3d_oracle_block* b);
void e3d_oracle_halo(e3d_oracle_block* blocks, const e3d_oracle_connexion* c, int n_connexions);
/* out[0..4] = per-equation sum of (Rc-Rd)^2; out[5..9] = wall sums fy, fx, cmx, cmy, cmz */
void e3d_oracle_flow_data(const e3d_oracle_block* b, const e3d_oracle_params* p, double out[10]);
/* n outer iterations over all blocks (Solver::solve body); hist[it*15 + ...] =
 * rms[5], cl, cd, cmx, cmy, cmz, conv[5] (rms0 taken from *rms0 when have_rms0,
 * else from the first iteration, and written back) */
int e3d_oracle_iterate(e3d_oracle_block* blocks, int n_blocks, const e3d_oracle_connexion* c, int n_connexions,
                       const e3d_oracle_params* p, int n_iter, int first_iter, double* rms0, int* have_rms0,
                       double* hist);
/* FP32 model library only (libe3d_oracle32.so): with a nonzero seed every
 * face flux is left as computed (half the cases) or moved one FP32 unit up or
 * down (a quarter each), by a seeded hash (0: no perturbation; the FP64
 * library ignores the seed) */
void e3d_oracle_set_noise(unsigned long long seed);

#ifdef __cplusplus
}
#endif
#endif
