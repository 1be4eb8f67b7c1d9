/*
 * vlasov1d2v.h -- C ABI of the B200 (sm_100a) hot path of a 1D2V DG Vlasov-Poisson solver.
 *
 * Drop-in boundary for crewsdw/Vlasov1D2V's hot path: the semi-discrete DG right-hand side
 * (main/fluxes.py), the SSP-RK3 loop (main/timestep.py), the zeroth velocity moment
 * (main/grid.py) and the high-order-DFT Poisson solve (main/elliptic.py).  The reference
 * binds these as Python classes over CuPy; the Python host layer of this project
 * (vlasov1d2v_b200/) keeps those classes' signatures and calls the functions below through
 * ctypes.
 *
 * Conventions
 *   - Every state array is the reference's ghost-inclusive layout, C order:
 *       f[X][n][U][n][V][n],  X = nx + 2, U = nu + 2, V = nv + 2
 *     (main/grid.py:262-268).  Element index 0 and X-1 (U-1, V-1) are ghost elements.
 *   - FP64 contexts take double* states, FP32 contexts take float* states (void* below).
 *     Fields (E, phi, rho), energies and dt are always double.
 *   - All pointers passed to compute entry points are DEVICE pointers unless the name says
 *     host.  The library never allocates or frees caller buffers; it borrows them for the
 *     duration of the call.  The context owns only its immutable coefficient tables.
 *   - Work is enqueued on the caller's CUDA stream (cudaStream_t passed as void*; NULL =
 *     legacy default stream).  Entry points do not synchronise the device, except
 *     vl_ctx_create / vl_ctx_destroy (table upload / free).
 *   - Every entry point returns an int status (VL_OK = 0; negative = error) and never
 *     aborts the process.  vl_last_error() returns a message for the calling thread.
 */
#ifndef VLASOV1D2V_H
#define VLASOV1D2V_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VL_ABI_VERSION 2

#if defined(__GNUC__)
#define VL_API __attribute__((visibility("default")))
#else
#define VL_API
#endif

enum vl_status {
    VL_OK = 0,
    VL_ERR_INVALID = -1,     /* bad shape, order, null pointer or argument */
    VL_ERR_CUDA = -2,        /* a CUDA runtime call failed (message in vl_last_error) */
    VL_ERR_NONFINITE = -3,   /* a non-finite density / field / energy was detected */
    VL_ERR_UNSUPPORTED = -4, /* order or precision not compiled in */
    VL_ERR_TOO_LARGE = -5    /* a size exceeds a fixed capacity of the entry point */
};

enum vl_precision { VL_FP64 = 0, VL_FP32 = 1 };

/* x-halo convention of the RHS (main/fluxes.py:164-174 rolls over the ghost-inclusive axis):
 *   VL_XHALO_GHOST    read the x-ghost slabs of the input (reference semantics for a raw
 *                     semi_discrete_rhs call on an arbitrary array);
 *   VL_XHALO_PERIODIC wrap to the opposite interior slab (what the stepper's ghost sync,
 *                     main/timestep.py:143 and :167-168, makes equivalent).               */
enum vl_xhalo { VL_XHALO_GHOST = 0, VL_XHALO_PERIODIC = 1 };

/* Problem description.  Host pointers; copied into the context by vl_ctx_create. */
typedef struct vl_config {
    int32_t abi_version;      /* = VL_ABI_VERSION */
    int32_t precision;        /* enum vl_precision */
    int32_t nx, nu, nv;       /* interior element counts (Grid1D.res, main/grid.py:14) */
    int32_t n;                /* LGL nodes per element, 1..10 (Basis1D.order) */
    int32_t n_modes;          /* M = number of DFT wave numbers (main/grid.py:46-48) */
    int32_t reserved0;
    double accel;             /* electron acceleration multiplier (main/reference.py:61) */
    double bfield;            /* magnetic field B (Elliptic.magnetic_field) */
    double kappa;             /* Poisson coefficient (main/reference.py:63) */
    double jx, ju, jv;        /* element Jacobians 2/dx (main/grid.py:23) */
    double dx, du, dv;        /* element widths (main/grid.py:20) */
    double length_x;          /* x-domain length L (main/grid.py:19) */
    double umax, vmax;        /* max |node coordinate| incl. ghosts (main/grid.py:32) */
    double courant;           /* Courant number (main/timestep.py:78-79) */
    const double *up;         /* [n][n]   internal-flux matrix (main/basis.py:176-188) */
    const double *xi;         /* [n][2]   lift columns of the inverse mass (main/basis.py:110) */
    const double *xw;         /* [n]      LGL weights (Grid1D.quad_weights row, main/grid.py:26) */
    const double *u_nodes;    /* [(nu+2)*n] ghost-inclusive u coordinates (Grid1D.arr) */
    const double *v_nodes;    /* [(nv+2)*n] ghost-inclusive v coordinates */
    const double *wave_numbers; /* [M] */
    /* The high-order DFT in factored form (complex, interleaved re/im).  The reference's tensor
     * is their product, T[e, j, m] = dft_phase[e][m] dft_ell[j][m] (Grid1D.spectral_transform,
     * main/basis.py:204-228), and its inverse phases exp(i k_m x_{e,j}) (Grid1D.grid_phases,
     * main/grid.py:50) are conj(dft_phase[e][m]) dft_qnode[j][m].                            */
    const double *dft_ell;    /* [n][M]  Fourier transform of the nodal basis (ell_tilde) */
    const double *dft_phase;  /* [nx][M] exp(-i k_m mid_e), mid_e the element midpoints */
    const double *dft_qnode;  /* [n][M]  exp(i k_m (x_{e,j} - mid_e)) */
} vl_config;

typedef struct vl_ctx vl_ctx;

/* Device-resident loop state of the SSP-RK3 driver (Stepper.main_loop, main/timestep.py:81-139).
 * The caller allocates it (device memory, 64-byte aligned) and initialises it with
 * vl_run_state_init.  Kernels read and update it, so the loop runs without host syncs.     */
typedef struct vl_run_state {
    double dt;          /* dt of the running step (Stepper.dt) */
    double dt_next;     /* dt computed after stage 2 (main/timestep.py:184-185) */
    double time;        /* Stepper.time; advanced by the NEW dt after each step (ts:98) */
    double final_time;  /* the loop ends once time >= final_time (ts:91) */
    int64_t steps;      /* Stepper.steps_counter */
    int64_t max_steps;  /* the loop also ends once steps >= max_steps */
    int32_t active;     /* the step in flight runs (set at its first kernel) */
    int32_t active_next;/* whether the next step runs */
    int32_t status;     /* 0 ok; bit 0: non-finite density/field/energy */
    int32_t hist_capacity; /* ring size of the history arrays */
    double *energy_hist;/* [hist_capacity] field energy after step s at [s % cap] (ts:102-103) */
    double *time_hist;  /* [hist_capacity] time after step s */
    double *dt_hist;    /* [hist_capacity] dt after step s */
    double reserved[4];
} vl_run_state;

/* ---- context ------------------------------------------------------------------------- */
VL_API int vl_ctx_create(const vl_config *cfg, vl_ctx **out);
VL_API int vl_ctx_destroy(vl_ctx *ctx);
VL_API const char *vl_last_error(void);
VL_API int vl_abi_version(void);

/* number of elements of one ghost-inclusive state array: (nx+2) n (nu+2) n (nv+2) n */
VL_API size_t vl_state_elems(const vl_ctx *ctx);
/* bytes of scratch vl_ssp_rk3_steps needs (caller allocates, 256-B aligned): the moment
 * partials of the stage kernels                                                             */
VL_API size_t vl_workspace_bytes(const vl_ctx *ctx);

/* ---- hot-path operators ------------------------------------------------------------------ */

/* DGFlux.semi_discrete_rhs (main/fluxes.py:59-105): out[interior] = J_x F_x + J_u F_u + J_v F_v
 * for the ghost-inclusive state f with field E[(nx+2)][n] (main/elliptic.py:132-145).
 * Ghost rows of out are not written (the reference discards them).                        */
VL_API int vl_rhs(vl_ctx *ctx, const void *f, const double *E, void *out, int xhalo, void *stream);

/* The same operator with caller-chosen direction weights: out = w[0] F_x + w[1] F_u + w[2] F_v.
 * w = {1, 0, 0}, {0, 1, 0}, {0, 0, 1} give DGFlux.x_flux / u_flux / v_flux (main/fluxes.py:107-153),
 * which return the flux divergence of one direction without its Jacobian.                  */
VL_API int vl_rhs_weighted(vl_ctx *ctx, const void *f, const double *E, void *out, int xhalo,
                    const double *w_host, void *stream);

/* Distribution.moment_zero / moment_zero_of_arr (main/grid.py:303-321):
 * rho[nx][n] = sum over interior velocity nodes of f w_u w_v / (J_u J_v).                   */
VL_API int vl_moment(vl_ctx *ctx, const void *f, double *rho, void *stream);

/* Elliptic.poisson2 (main/elliptic.py:117-145): spectral solve of the charge density
 * (already mean-subtracted by the caller, as main/timestep.py:155 does).  Writes
 * E[(nx+2)][n] (ghosts periodic) and phi[nx][n] (phi may be NULL).  The mode coefficients
 * pass through a scratch owned by the context: calls on one context must not overlap.      */
VL_API int vl_poisson(vl_ctx *ctx, const double *charge_density, double *E, double *phi,
               void *stream);

/* Elliptic.electric_energy (main/elliptic.py:150-151): 0.5 sum_i w_i E[1:-1]^2 -> *energy. */
VL_API int vl_field_energy(vl_ctx *ctx, const double *E, double *energy, void *stream);

/* get_max_speeds + Stepper.adapt_time_step (main/timestep.py:231-242) from E -> *dt.       */
VL_API int vl_adapt_dt(vl_ctx *ctx, const double *E, double *dt, void *stream);

/* One fused SSP-RK stage (main/timestep.py:157-163 and :174-182):
 *   stage 0:  out = in + dt * RHS(in)                       (in is f^n)
 *   stage 1:  out = 3/4 fn + 1/4 in + 1/4 dt RHS(in)
 *   stage 2:  out = 1/3 fn + 2/3 in + 2/3 dt RHS(in)
 * dt is read from device memory (*dt).  Interior of out only.  If workspace is not NULL the
 * stage also writes the moment partials of out (per x element, one partial density row per
 * CTA; the loop's field solve sums them).                                                    */
VL_API int vl_rk_stage(vl_ctx *ctx, int stage, const void *in, const void *fn, void *out,
                const double *E, const double *dt, int xhalo, void *workspace, void *stream);

/* ---- the loop ------------------------------------------------------------------------------ */

/* Fill a device vl_run_state: dt from E0 (adapt rule), time 0, steps 0, histories given.
 * E0 is the field solved before the loop (main/main.py:131); its energy is returned in
 * *energy0 (device pointer, may be NULL).                                                    */
VL_API int vl_run_state_init(vl_ctx *ctx, vl_run_state *state, const double *E0, double final_time,
                      int64_t max_steps, double *energy_hist, double *time_hist,
                      double *dt_hist, int32_t hist_capacity, double *energy0, void *stream);

/* Stepper.nonlinear_ssp_rk x nsteps (main/timestep.py:141-187) with the main loop's
 * bookkeeping (ts:91-103), entirely on the device: each step runs only while
 * state->time < final_time and steps < max_steps (checked on the device, so extra steps
 * in a batch are no-ops).  f is advanced in place.  stage_a / stage_b are state-sized
 * buffers whose velocity-ghost elements must equal f's (vl_sync_ghosts does that).
 * E / phi receive the last field solved (of RK stage s1, as in the reference).             */
VL_API int vl_ssp_rk3_steps(vl_ctx *ctx, void *f, void *stage_a, void *stage_b, double *E,
                     double *phi, vl_run_state *state, void *workspace, int nsteps,
                     void *stream);

/* No counterpart in the reference (the FP32 mixed form).  Background split: the FP32 state
 * holds delta f = f - f0(u, v), f0 an x-independent background kept in FP64 on the host side,
 * so the x derivative no longer cancels the O(1) background against the O(1e-3) perturbation
 * in FP32.  The stage kernels then add the RHS of f0 per node,
 *   r0 = E_i eu + rb,
 * with rb = J_u a B v D_u f0 + J_v (-a B u) D_v f0 and eu = J_u a D_u f0 precomputed in FP64
 * and stored as float in the velocity-slab layout [(nu+2)][n][(nv+2)][n] (device pointers,
 * 16-byte aligned, caller-owned, kept until the next call).  f0 is continuous across element
 * faces, so its upwind and downwind face traces agree and one D_u table serves both signs of
 * the u speed.  The x contraction of f0 is zero (f0 is constant in x).  Pass two NULLs to switch
 * the split off.  FP32 contexts only.                                                         */
VL_API int vl_set_background(vl_ctx *ctx, const float *rb, const float *eu);

/* Optional, with vl_set_background: the same two tables interleaved per column pair,
 *   pairs[r][p] = {eu[r][2p], eu[r][2p+1], rb[r][2p], rb[r][2p+1]},  r over the (nu+2) n rows,
 * p over the (nv+2) n / 2 column pairs (16-byte aligned, caller-owned, kept until the next call).
 * The order-8 FP32 stage kernel then stages both tables with one tensor copy and reads them with
 * one 128-bit load per row.  NULL clears it; vl_set_background(ctx, NULL, NULL) clears it too.
 * FP32 contexts with an even (nv+2) n only.                                                     */
VL_API int vl_set_background_pairs(vl_ctx *ctx, const float *pairs);

/* Copy f's ghost elements (all six ghost slabs) into a stage buffer and perform the
 * reference's periodic x-ghost swap on f (Distribution.swap_ghost_cells_of_array,
 * main/grid.py:187-189).  Call once before a run and after f is replaced.                  */
VL_API int vl_sync_ghosts(vl_ctx *ctx, void *f, void *stage, void *stream);

/* ---- the DG Poisson solve and the linear SSP-RK stepper's interior update ------------------- */

/* Elliptic.poisson (main/elliptic.py:85-115): stabilised central-flux DG solve of the
 * mean-subtracted charge density.  inv_op = the inverse of the bordered operator
 * [(nx n + 1)^2] (Elliptic.invert), mass = the element mass matrix [n][n], grad_op = the
 * gradient operator [nx n][nx n] (G[q][p]), all device tables of the host set-up
 * (main/elliptic.py:24-83); anti_alias != 0 filters the potential and the field through the
 * context's high-order DFT.  Writes E[(nx+2)][n] (periodic ghosts) and phi[nx][n] (may be NULL).
 * One CTA: nx n up to about 8000.                                                              */
VL_API int vl_poisson_dg(vl_ctx *ctx, const double *charge_density, const double *inv_op,
                         const double *mass, const double *grad_op, int32_t anti_alias, double *E,
                         double *phi, void *stream);

/* y[interior] <- alpha y[interior] + beta x[interior] (x may be NULL: beta ignored); ghost
 * elements untouched.  The accumulation of Stepper.ssp_rk_update (main/timestep.py:195, :213). */
VL_API int vl_axpby_interior(vl_ctx *ctx, void *y, const void *x, double alpha, double beta,
                             void *stream);

/* ---- around the loop: initial state, post-processing ------------------------------------------
 * These take the grid dimensions and state precision directly (no context): they need none of
 * the context's tables.  prec is VL_FP64 or VL_FP32; arithmetic is FP64 in both. */

/* Distribution.initialize_gpu (main/grid.py:244-279) and the eigenmode perturbation
 * (main/grid.py:201-242), the O(DOF) part on the device:
 *   f[e,i,a,j,b,k] = pol[a,j,b,k] * mx[e,i] + scale * (cx[e,i] vre[a,j,b,k] - sx[e,i] vim[a,j,b,k])
 * pol = the loss-cone values factor * rsq^j exp(-rsq/2) on the velocity nodes incl. ghosts
 * [(nu+2) n (nv+2) n]; mx = an x-node factor [(nx+2) n] or NULL (1); vre/vim = the eigenmode's
 * velocity part (real, imaginary), cx/sx = cos/sin(k1 x) [(nx+2) n], scale = 2 delta_n; vre
 * NULL = no perturbation.  The O(velocity) tables come from the host (Bessel series). */
VL_API int vl_initial_state(void *f, int32_t prec, int32_t nx, int32_t nu, int32_t nv, int32_t n,
                            const double *pol, const double *mx, const double *cx,
                            const double *sx, const double *vre, const double *vim, double scale,
                            void *stream);

/* smooth_edges (main/grid.py:116-134): in place, the face-node planes of every interior element
 * averaged with the neighbour's opposite face, x then u then v, left then right.  n >= 2. */
VL_API int vl_smooth_edges(void *f, int32_t prec, int32_t nx, int32_t nu, int32_t nv, int32_t n,
                           void *stream);

/* Basis3D.interpolate_values (main/basis.py:291-317): values of the nodal polynomials on fine
 * points of the elements lims = {x0, x1, u0, u1, v0, v1} (ghost-inclusive element indices,
 * interior only, half-open).  ell_x[ex][n][fx] (ell_u, ell_v likewise) are the Lagrange
 * polynomials at the fine points of each element of the range (host tables of the reference's
 * construction); out[ex][fx][eu][fu][ev][fv] (FP64).  At most 32 fine points per element. */
VL_API int vl_interpolate(const void *f, int32_t prec, int32_t nx, int32_t nu, int32_t nv,
                          int32_t n, const int32_t *lims, const double *ell_x, const double *ell_u,
                          const double *ell_v, int32_t fx, int32_t fu, int32_t fv, double *out,
                          void *stream);

/* ---- batched heterogeneous ensemble ------------------------------------------------------------
 * No counterpart in the reference (which runs one problem per process).  Many independent
 * problems -- each an ordinary context of any order 1..9 and grid, one common precision --
 * advance together: per RK stage one forward-DFT launch, one inverse-DFT launch and persistent
 * stage kernels (one for all members, or one per order present) whose CTAs walk host-built lists
 * of (member, x element, tile group) work items balanced by estimated cost.  Members keep their own
 * loop state (final time, histories); inactive members are skipped on the device.
 *   vl_ens_create     members = existing contexts (borrowed; keep them alive)
 *   vl_ens_bind       member i's state f, stage buffers, E, phi, loop state and workspace of
 *                     vl_ens_workspace_bytes(ens, i) bytes (the stage buffers' velocity ghosts
 *                     must equal f's, as for vl_ssp_rk3_steps)
 *   vl_ens_schedule   tunables: threads per CTA (64 or 128), resident CTAs per SM, work items
 *                     per CTA (tile groups per x slab follow from it)
 *   vl_ens_schedule_by_order
 *                     alternative schedule: one stage launch per order present, each kernel
 *                     built for its order alone (as many CTAs as stay resident, work items per
 *                     CTA), except for the orders whose bit n is set in native_orders: their
 *                     members are launched one by one through their own context's stage kernel
 *                     (the single-problem kernel choice, e.g. the tensor-core one for n = 8);
 *                     VL_ENS_NATIVE_AUTO picks the members whose contexts stage their tiles by
 *                     TMA; the launches of one stage run on concurrent streams
 *   vl_ens_commit     upload descriptors and the item list (synchronous; not inside a capture)
 *   vl_ens_steps      nsteps SSP-RK3 steps of every member (stream-ordered, capturable)      */
typedef struct vl_ens vl_ens;
#define VL_ENS_NATIVE_AUTO 0xFFFFFFFFu
VL_API int vl_ens_create(vl_ctx *const *ctxs, int32_t count, vl_ens **out);
VL_API int vl_ens_destroy(vl_ens *ens);
VL_API size_t vl_ens_workspace_bytes(const vl_ens *ens, int32_t i);
VL_API int vl_ens_bind(vl_ens *ens, int32_t i, void *f, void *stage_a, void *stage_b, double *E,
                       double *phi, vl_run_state *state, void *workspace);
VL_API int vl_ens_schedule(vl_ens *ens, int32_t threads, int32_t ctas_per_sm, int32_t items_per_cta);
VL_API int vl_ens_schedule_by_order(vl_ens *ens, int32_t items_per_cta, uint32_t native_orders);
VL_API int vl_ens_commit(vl_ens *ens);
VL_API int vl_ens_steps(vl_ens *ens, int32_t nsteps, void *stream);

/* ---- learned coarse-grid closure ------------------------------------------------------------------
 * No counterpart in the reference.  A per-(x node, velocity element) MLP corrects the RHS of a
 * coarse (order 6) velocity grid towards the L2 projection of a fine-grid RHS.
 * Network: IN = 96 inputs -> 128 -> 128 -> 128 (GELU) -> OUT = 48 outputs (first 36 used),
 * bf16 weights and activations, FP32 accumulation (tensor cores, mma m16n8k16).  Weights live
 * in two bf16 layouts, wf = [out][in] and wb = [in][out] per layer, layers back to back
 * (layer offsets 0, 96*128, 96*128 + 128*128, 96*128 + 2*128*128; n_weights elements), and
 * FP32 biases (offsets 0, 128, 256, 384; n_bias elements); vl_mlp_dims reports the sizes.    */
VL_API int vl_mlp_dims(int32_t *in, int32_t *hidden, int32_t *out, int32_t *n_weights, int32_t *n_bias);
/* Y[nrows][48] = MLP(X[nrows][96]).  With H0 [nrows][96] bf16, Hh [3][nrows][128] bf16 and
 * Z [3][nrows][128] FP32 given, the layer inputs and hidden pre-activations are kept for
 * vl_mlp_backward (all three or none).                                                      */
VL_API int vl_mlp_forward(const float *X, int32_t nrows, const void *wf, const void *wb, const float *bias,
                          float *Y, void *H0, void *Hh, float *Z, void *stream);
/* FP32 elements of the per-block gradient partials vl_mlp_backward needs for nrows samples. */
VL_API size_t vl_mlp_partial_floats(int32_t nrows);
/* Gradient of L = sum_{rows, c < nout} (Y - T)^2 / (nrows nout), T[nrows][nout], through the
 * network (bf16 operands, FP32 accumulation; per-block partials summed in a fixed order):
 * grad_w in the [in][out] layout, grad_b.                                                    */
VL_API int vl_mlp_backward(const float *Y, const float *T, int32_t nrows, int32_t nout, const void *wf,
                           const void *wb, const float *bias, const void *H0, const void *Hh, const float *Z,
                           float *partials, float *grad_w, float *grad_b, void *stream);
/* One Adam step (step >= 1: bias corrections) on FP32 master weights ([in][out]) and biases,
 * with decoupled weight decay; refreshes both bf16 layouts.                                   */
VL_API int vl_mlp_adam(float *master_w, float *master_b, const float *grad_w, const float *grad_b, float *m_w,
                       float *v_w, float *m_b, float *v_b, void *wf, void *wb, float lr, float beta1,
                       float beta2, float eps, int32_t step, float weight_decay, void *stream);
/* Closure inputs of a coarse state f (order 6): one sample per (x node, interior velocity
 * element), X[nx*6*nu*nv][96] (84 state values divided by the sample's scale max|.|, then
 * a E_i / escale, u / umax and v / vmax of the element centre, a B, zeros), scale[samples].  */
VL_API int vl_closure_features(const void *f, int32_t prec, int32_t nx, int32_t nu, int32_t nv,
                               const double *E, double accel, double bfield, const double *u_nodes,
                               const double *v_nodes, double umax, double vmax, double escale, float *X,
                               float *scale, void *stream);
/* out[e, i, a, j, b, k] += c2 * (*dt) * cscale * c[s, j, k], c = scale[s] * clamp(Y[s][6 j + k],
 * +-ymax), for every interior node: the network's RHS correction applied to an RK stage output,
 * its outputs clamped to the range seen in training (state may be NULL; an inactive loop state
 * skips it).  mode VL_CLOSURE_CHARGE subtracts from c, per x node, its quadrature mean over all
 * velocity nodes (weights node_weights[j] node_weights[k], the 6 LGL weights; host pointer), so
 * the correction conserves the charge density the field is solved from.                        */
enum vl_closure_mode { VL_CLOSURE_PLAIN = 0, VL_CLOSURE_CHARGE = 1 };
VL_API int vl_closure_apply(void *out, int32_t prec, int32_t nx, int32_t nu, int32_t nv, const float *Y,
                            const float *scale, double cscale, float ymax, const double *dt, double c2,
                            const vl_run_state *state, int32_t mode, const double *node_weights,
                            void *stream);

/* ---- the loop without a caller-provided workspace ------------------------------------------- */

/* No counterpart in the reference.  vl_ssp_rk3_steps for callers that cannot allocate device
 * memory themselves -- e.g. a host recording the loop into a CUDA graph while allocation is
 * not allowed, a plugin whose host framework owns the whole device heap, or a binding that
 * holds only raw buffer pointers and a stream.  Same arguments and results as
 * vl_ssp_rk3_steps minus the workspace: the loop's scratch is a file-scope device array
 * of VL_NOALLOC_SCRATCH_BYTES inside the library (every GPU that loads the library holds it
 * until the process exits).  Problems whose vl_workspace_bytes exceeds that size are rejected
 * with VL_ERR_TOO_LARGE (the scratch of the problems the kernels accept -- nx n <= 640 -- stays
 * below 100 KB).  Call it with the context's device current (another device is rejected with
 * VL_ERR_INVALID).  The first call on a device looks the array's address up with that device
 * current; make it before any stream capture.  The address is cached for the life of the
 * process: after a cudaDeviceReset do not call this entry point again on that device.  All calls share the array and it keeps
 * the last call's contents (the loop writes every entry it reads before reading it), so calls
 * whose kernels overlap on the GPU race on it.  Nothing here calls cudaMalloc or cudaFree.     */
#define VL_NOALLOC_SCRATCH_BYTES (1u << 20)
VL_API int vl_ssp_rk3_steps_noalloc(vl_ctx *ctx, void *f, void *stage_a, void *stage_b, double *E,
                                    double *phi, vl_run_state *state, int nsteps, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* VLASOV1D2V_H */
