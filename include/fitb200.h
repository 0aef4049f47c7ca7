/*
 * fitb200.h -- C ABI of the B200-native FIT-TD (Yee leapfrog) time-stepping
 * engine behind Magnelio's FITTimeDomainSolver.
 *
 * Conventions
 *   - Every function returns an int status: FITB_OK (0) or a negative
 *     FITB_ERR_* code.  fitb_last_error() returns the message of the most
 *     recent failure on the calling thread.
 *   - Host pointers are borrowed for the duration of the call only.  All
 *     device memory is owned by the handle and released by fitb_destroy().
 *   - Array layouts are the reference's: the flat E vector is
 *     [Ex | Ey | Ez] with Ex (Nx, Ny+1, Nz+1), Ey (Nx+1, Ny, Nz+1),
 *     Ez (Nx+1, Ny+1, Nz); the flat H vector is [Hx | Hy | Hz] with
 *     Hx (Nx+1, Ny, Nz), Hy (Nx, Ny+1, Nz), Hz (Nx, Ny, Nz+1); C order,
 *     k (z) fastest  (reference: src/magnelio/_fields/field_arrays.py:1-17).
 *   - Field buffers passed by the caller have the handle's precision
 *     (float32 when precision == 4, float64 when precision == 8).
 *     Setup constants (coefficients, profiles, CPML tables, waveform
 *     samples) are passed as float64 and rounded once on upload, as the
 *     reference builds them in float64 and casts
 *     (reference: src/magnelio/solver/fit_td.py:468-479).
 *   - One CUDA stream per handle; calls on one handle are not thread-safe.
 *   - A handle carries B field sets ("batch") that share one coefficient set;
 *     every per-field-set argument takes the field-set index b in [0, B).
 */
#ifndef FITB200_H
#define FITB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FITB_ABI_VERSION 1

#define FITB_OK 0
#define FITB_ERR_ARG (-1)      /* invalid argument / size mismatch          */
#define FITB_ERR_CUDA (-2)     /* CUDA runtime error                         */
#define FITB_ERR_STATE (-3)    /* call not valid in the handle's state      */
#define FITB_ERR_NOMEM (-4)    /* device allocation failed                   */
#define FITB_ERR_NODEV (-5)    /* no usable CUDA device                      */
#define FITB_ERR_LIMIT (-6)    /* a fixed capacity of the engine exceeded    */

typedef struct fitb_handle fitb_handle;

/* Grid and run description.  Replaces the mesh / dt / precision fields of
 * FITTimeDomainSolver (reference: src/magnelio/solver/fit_td.py:174-234,
 * setup at :302-324). */
typedef struct fitb_desc {
    int32_t nx, ny, nz;   /* cell counts                                    */
    int32_t batch;        /* field sets sharing the coefficients (>= 1)     */
    int32_t precision;    /* 4 = float32 fields, 8 = float64 fields         */
    int32_t device;       /* CUDA device ordinal                            */
    double dt;            /* time step [s]                                  */
} fitb_desc;

/* Modal (waveguide) port.  Mirrors PortOperatorModal's per-step data
 * (reference: src/magnelio/ports/_modal/operator.py:510-640 constructor,
 * :1351-1536 update_e, :1253-1321 projections).  All index arrays are flat
 * indices into the reference E or H vector.  The interior plane has the
 * same (u, v) sample counts as the port plane. */
typedef struct fitb_modal_desc {
    int32_t n_modes;
    int32_t n_e_u, n_e_v;        /* port-plane E samples, u then v           */
    int32_t n_h_u, n_h_v;        /* port-plane dual-edge H samples           */
    const int64_t* port_e_idx;   /* [n_e_u + n_e_v]   plane.e_u/e_v_indices   */
    const int64_t* int_e_idx;    /* [n_e_u + n_e_v]   interior plane indices  */
    const int64_t* port_h_idx;   /* [n_h_u + n_h_v]   plane.h_u/h_v_indices   */
    const double* me_port;       /* [n_e_u + n_e_v]   M_eps at port plane     */
    const double* me_int;        /* [n_e_u + n_e_v]   M_eps at interior plane */
    const double* mh_port;       /* [n_h_u + n_h_v]   M_mu at port dual edges */
    const double* e_profile;     /* [n_modes][n_e]    reconstruction profile  */
    const double* v_profile;     /* [n_modes][n_e]    projection profile (dual basis, or primal) */
    const double* h_profile;     /* [n_modes][n_h]    current profile         */
    const double* mur_r;         /* [n_modes]                                 */
    const double* tau;           /* [n_modes]  TF/SF delay tau_m [s]          */
    const double* record_scale;  /* [n_modes]                                 */
    const int32_t* is_dtbc;      /* [n_modes]  1: exact DTBC, 0: modal Mur    */
    const double* dtbc_r;        /* [n_modes]                                 */
    const double* dtbc_q;        /* [n_modes]                                 */
    int32_t dtbc_n_kernel_init;  /* initial kernel length (power of two)      */
    int32_t has_complement;      /* complement absorber configured            */
    const double* comp_r;        /* [n_e] per-edge Mur coefficient            */
    const double* comp_live;     /* [n_e] 0/1 live mask                       */
    int64_t max_steps;           /* history capacity in steps                 */
} fitb_modal_desc;

/* Running-DFT field monitor over a cell box (reference:
 * src/magnelio/monitors/field_frequency.py:249-294 record,
 * src/magnelio/monitors/base.py:51-168 cell-centre interpolation,
 * src/magnelio/monitors/_dft.py:37-52 accumulate). */
typedef struct fitb_dft_desc {
    int32_t i0, i1, j0, j1, k0, k1;  /* cell-index box, stop-exclusive      */
    int32_t comp_mask;               /* bit c set = record component c,
                                        c = 0..5 for Ex,Ey,Ez,Hx,Hy,Hz      */
    int32_t n_freq;
    const double* freqs;             /* [n_freq] Hz                          */
    int32_t stride;                  /* record every stride-th step (>= 1)   */
    int32_t kahan;                   /* 1: compensated float32 bins          */
    const double* dx;                /* [nx] primal widths                   */
    const double* dy;                /* [ny]                                 */
    const double* dz;                /* [nz]                                 */
} fitb_dft_desc;

/* TF/SF plane-wave source (sources/plane_wave.py:65-733): ordered face
 * patches as flat indices into the reference's e_flat / h_flat, each entry
 * with its coefficient (beta * metric * incident amplitude, already rounded
 * to the field dtype) and retardation delay [s].  After the E update of
 * step n every E entry gets coef * f(n dt + dt - dt/2 - delay) added, after
 * the H update every H entry coef * f(n dt + dt + dt/2 - dt/2 - delay);
 * entries that appear more than once take their contributions in the order
 * given.  f(t) = amplitude * exp(-((t - t0)^2) / den)   (FITB_WAVE_GAUSSIAN)
 *        f(t) = amplitude * sin(omega t)                 (FITB_WAVE_SINE). */
#define FITB_WAVE_GAUSSIAN 0
#define FITB_WAVE_SINE 1
typedef struct fitb_plane_wave_desc {
    int32_t waveform;
    double amplitude, t0, den, omega;
    int64_t n_e;
    const int64_t* e_idx;
    const double* e_coef;
    const double* e_delay;
    int64_t n_h;
    const int64_t* h_idx;
    const double* h_coef;
    const double* h_delay;
} fitb_plane_wave_desc;

/* ---- lifetime ------------------------------------------------------- */
/* FITB_ABI_VERSION of the built library; a binding compares it with the
 * header it was written against (no counterpart in the reference). */
int fitb_abi_version(void);
/* Replaces FITTimeDomainSolver.setup() allocation (fit_td.py:302-324). */
int fitb_create(const fitb_desc* desc, fitb_handle** out);
/* Frees the handle and all device memory it owns (the reference drops its
 * arrays with the solver object). */
int fitb_destroy(fitb_handle* h);
/* Message of the most recent failed call, NUL-terminated into buf (the
 * reference raises exceptions; the binding turns a non-zero status and
 * this message into one). */
int fitb_last_error(char* buf, size_t len);
/* Number of this library's kernel launches issued so far on the handle. */
int fitb_launch_count(const fitb_handle* h, int64_t* out);

/* ---- coefficients and fields ---------------------------------------- */
/* alpha/beta of the leapfrog update and the mass diagonals for the energy
 * check (fit_td.py:383-514).  Lengths n_E and n_H of the reference flat
 * layout.  m_eps / m_mu may be NULL (energy then reports 0). */
int fitb_set_coeffs(fitb_handle* h, const double* alpha_e, const double* beta_e,
                    const double* alpha_h, const double* beta_h,
                    const double* m_eps, const double* m_mu);
/* Same, with the arrays already in the field dtype (float32 / float64):
 * the reference casts its float64 build to the field dtype before the
 * march (fit_td.py:468-479), so its cast arrays upload as they are. */
int fitb_set_coeffs_native(fitb_handle* h, const void* alpha_e, const void* beta_e,
                           const void* alpha_h, const void* beta_h,
                           const void* m_eps, const void* m_mu);
/* Material matrices and leapfrog coefficients built on the device from the
 * grid and the cell materials, in place of fitb_set_coeffs for lossless,
 * non-magnetic problems (replaces the host-side setup of
 * FITTimeDomainSolver.setup, src/magnelio/solver/fit_td.py:341-514, over
 * build_M_eps / build_M_mu, src/magnelio/_operators/material_matrices.py
 * :334-531): dx, dy, dz the nx, ny, nz cell widths [m]; mat_id[nx][ny][nz]
 * the material of each cell (0 .. n_mat-1) and eps_r[n_mat] its relative
 * permittivity.  An E edge takes the permittivity of its owner cell (the
 * cell at its (i, j, k), clamped to the grid) times EPS0 A_dual / L_primal;
 * the n_cat1 edges cat1_idx (flat E indices) take cat1_eps instead (conformal
 * averages); M_mu = MU0 A_primal / L_dual; alpha = 1, beta = dt / M (M = 0:
 * frozen at (1, 0)); the n_pec edges pec_idx are frozen at (0, 0).  The
 * float64 arithmetic is rounded as written, so the result equals the host
 * restatement's bit for bit. */
int fitb_build_materials(fitb_handle* h, const double* dx, const double* dy, const double* dz, const int32_t* mat_id,
                         int32_t n_mat, const double* eps_r, int64_t n_cat1, const int64_t* cat1_idx,
                         const double* cat1_eps, int64_t n_pec, const int64_t* pec_idx);
/* Spectral time-step limit on the device (replaces the host Lanczos of
 * spectral_dt / _measure_lambda_max, src/magnelio/solver/stability.py
 * :296-446): lambda_max of D^-1/2 C^T M_mu^-1 C D^-1/2 (D = M_eps) on the
 * live E edges (beta_E != 0, M_eps > 0), measured matrix-free by a float64
 * Lanczos iteration on the handle's M_eps, M_mu and beta_E (so after
 * fitb_set_coeffs with both mass diagonals, or fitb_build_materials), until
 * the largest Ritz value changes by less than tol (relative) over ten steps
 * or after max_iter steps; dt = safety * 2 / sqrt(lambda_max) (the reference's
 * safety factors: 0.95 "normal").  A float32 handle holds its mass diagonals
 * in float32, which limits lambda_max to float32 accuracy; a float64 handle
 * reproduces the reference's value to the Lanczos tolerance.  iterations
 * (may be NULL) receives the steps taken. */
int fitb_spectral_dt(fitb_handle* h, double safety, int32_t max_iter, double tol, double* lambda_max, double* dt,
                     int32_t* iterations);
/* Storage of the four update-coefficient arrays read by the stream stencil
 * kernels: FITB_COEF_NATIVE (field dtype, the default), FITB_COEF_F16 or
 * FITB_COEF_BF16 (16-bit values with a power-of-two scale per component;
 * the arithmetic stays in the field dtype).  The compact forms change the
 * coefficients by their 16-bit rounding (relative 2^-11 for float16,
 * 2^-8 for bfloat16), so the march is no longer the reference's to
 * round-off; they halve the coefficient reads (96 -> 72 bytes per cell and
 * step in float32).  No counterpart in the reference, which stores the
 * coefficients in the field dtype (fit_td.py:468-479).  Valid before or
 * after fitb_set_coeffs; FITB_ERR_STATE when the handle does not use the
 * stream kernels. */
#define FITB_COEF_NATIVE 0
#define FITB_COEF_F16 1
#define FITB_COEF_BF16 2
int fitb_set_coeff_storage(fitb_handle* h, int32_t kind);
/* Stencil form of the handle (no counterpart in the reference, whose kernels
 * are fixed): kind FITB_STENCIL_SIMPLE / STREAM / BULK / VEC / FUSED, a
 * variant of that form (vec 0-3; fused 0-6 the register / cp.async forms,
 * fused 7-15 the TMA tile form with its CPML slab passes, tile shapes of
 * 2-16 rows x 32 cells and 3-5 ring stages; fused 16-25 the slab step, the
 * TMA tile march with the CPML inside it, tiles of 4, 2, 3, 4, 3, 2, 8, 6,
 * 4, 4 rows x 32 cells with 3, 3, 3, 4, 4, 4, 3, 3, 3, 3 ring stages, one
 * field set per CTA except 24 and 25, which march 2 and 4 field sets per
 * CTA through shared coefficient boxes (the batch a multiple of that);
 * 22 and 25 are float32 only (their shared memory exceeds a CTA's in
 * float64), and grids whose units reach both faces of an axis refuse the
 * forms without a six-slot kernel (25; 23 and 24 in float64);
 * FITB_ERR_ARG for a form the handle's
 * precision, dispersion or CPML layout does not take), and the number of i
 * planes one CTA marches (0: the form's own plan).  The fields, psi and all
 * other state carry over; valid between steps.
 * fitb_get_stencil writes kind, variant, planes per CTA and the grid
 * (x, y, z) into out[6]. */
#define FITB_STENCIL_SIMPLE 0
#define FITB_STENCIL_STREAM 1
#define FITB_STENCIL_BULK 2
#define FITB_STENCIL_VEC 3
#define FITB_STENCIL_FUSED 4
int fitb_configure_stencil(fitb_handle* h, int32_t kind, int32_t variant, int32_t ichunk);
int fitb_get_stencil(fitb_handle* h, int32_t* out);
/* Work units of the slab step (fused 16-25): out[0..4] the units launched
 * with 0, 1, 2, 3 and up to 6 CPML face slots, out[5] the units left out as
 * dead (every E edge frozen at zero, every H face a no-op or curl-dead; the
 * reference's tile skip, solver/_tile_skip.py:187, which this follows,
 * including its off switch with TF/SF plane waves; FITB_TILE_SKIP=0 turns
 * it off).  All zero in other forms. */
int fitb_slab_units(fitb_handle* h, int64_t* out);
/* Device memory the handle holds, in bytes (every buffer it allocated; the
 * recorder and DTBC histories grow with the step capacity). */
int fitb_device_bytes(fitb_handle* h, int64_t* out);
/* Size the recorder and DTBC histories for n_steps completed steps up front
 * (they otherwise grow by doubling, which re-captures the step graphs). */
int fitb_reserve_steps(fitb_handle* h, int64_t n_steps);
/* FieldState e_flat / h_flat of field set b (field_arrays.py:98-106). */
int fitb_set_fields(fitb_handle* h, int32_t b, const void* e, size_t e_bytes,
                    const void* hf, size_t h_bytes);
int fitb_read_fields(fitb_handle* h, int32_t b, void* e, size_t e_bytes,
                     void* hf, size_t h_bytes);

/* ---- boundaries ----------------------------------------------------- */
/* CFS-PML face (reference: src/magnelio/boundaries/cpml.py:92-195
 * initialize, :213-310 set_pec_mask, :343-516 update_E/update_H).
 * face: 0..5 = xmin,xmax,ymin,ymax,zmin,zmax.  b/c/ck: per-layer tables of
 * length n_pml.  air_*: 0/1 masks in the reference psi shapes
 * (e.g. z face: psi_Ex (Nx,Ny+1,n), psi_Ey (Nx+1,Ny,n), psi_Hx (Nx+1,Ny,n),
 * psi_Hy (Nx,Ny+1,n)); NULL = all ones. */
int fitb_add_cpml(fitb_handle* h, int32_t face, int32_t n_pml,
                  const double* b, const double* c, const double* ck,
                  const uint8_t* air_e1, const uint8_t* air_e2,
                  const uint8_t* air_h1, const uint8_t* air_h2);

/* ---- lumped ports --------------------------------------------------- */
/* Thevenin lumped element with a series R-L-C companion (reference:
 * src/magnelio/ports/_lumped/operator.py:134-166 update_e,
 * src/magnelio/circuit/companion.py SeriesRLC).  r, l, c < 0 = absent. */
int fitb_add_lumped(fitb_handle* h, int32_t n_edges, const int64_t* flat_e_idx,
                    const double* signs, const double* betas,
                    double r, double l, double c, double record_scale,
                    int32_t* out_id);
/* Source voltage samples v_src[n] = waveform((n+1)*dt) for steps
 * n = 0..n_samples-1 (zero beyond). */
int fitb_set_lumped_source(fitb_handle* h, int32_t id, int32_t b,
                           int64_t n_samples, const double* v_src);

/* Stream source samples into an existing table: v_src[step0 .. step0+n) of
 * field set b is overwritten by an asynchronous copy, on the handle's
 * stream, from `host` (which should be pinned memory and must stay valid
 * until the next fitb_sync / fitb_read_* call).  For co-simulation, where
 * the next step's source voltage is produced on the host while the device
 * steps.  The table must already be long enough (fitb_set_lumped_source). */
int fitb_push_lumped_samples(fitb_handle* h, int32_t id, int32_t b, int64_t step0,
                             int64_t n, const double* host);

/* ---- modal ports ---------------------------------------------------- */
int fitb_add_modal_port(fitb_handle* h, const fitb_modal_desc* d, int32_t* out_id);
/* DTBC convolution kernel l_m (m = 0..n_kernel-1) of mode `mode` for the
 * table length n_kernel (reference: src/magnelio/ports/_modal/dtbc.py:125-156,
 * auto-extension :351-363).  One call per power-of-two length. */
int fitb_set_dtbc_kernel(fitb_handle* h, int32_t port, int32_t mode,
                         int32_t n_kernel, const double* l);
/* The same tables built on the device (per-request setup): every length
 * n0, 2 n0, ... up to the first >= n_steps that is not set yet, from the
 * mode's r and q given to fitb_add_modal_port.  The Laurent coefficients
 * of the outgoing root are the inverse DFT of 8 n samples on the circle
 * |z| = exp(4 / n) (dtbc.py:125-156), summed directly in float64 on the
 * GPU: they agree with the reference's FFT to round-off, not bit for bit.
 * FITB_ERR_ARG for a mode that is not DTBC. */
int fitb_build_dtbc_kernel(fitb_handle* h, int32_t port, int32_t mode, int64_t n_steps);
/* Excite mode `mode` of field set b with waveform samples
 * w[n] = waveform(n*dt), n = 0..n_samples-1 (zero beyond); mode = -1 clears
 * (operator.py:1140-1182 set_excitation / clear_excitation). */
int fitb_set_modal_source(fitb_handle* h, int32_t port, int32_t b, int32_t mode,
                          int64_t n_samples, const double* w);

/* ---- dispersive materials ------------------------------------------- */
/* One dispersive material's ADE block (solver/_dispersion.py:173-210,
 * :504-569): side 0 = eps(omega) on E edges, 1 = mu(omega) on H faces;
 * n_states flat indices into the reference E (or H) vector with their
 * geometry factor g; per pole its kind (0 real, 1 conjugate pair stored
 * once), k = (1 + a dt/2)/(1 - a dt/2), c = r/(1 - a dt/2) (imaginary parts
 * ignored for real poles) and weight (1 or 2).  Blocks of one side are kept
 * in the order added; the alpha/beta already carry the W folding
 * (fit_td.py:383-399, :436-446).  Not valid in the fused step mode. */
int fitb_add_dispersion_block(fitb_handle* h, int32_t side, int64_t n_states, const int64_t* idx,
                              const double* g, int32_t n_poles, const int32_t* kind,
                              const double* k_re, const double* k_im, const double* c_re,
                              const double* c_im, const double* weight);

/* ---- band-subspace DTBC ports ---------------------------------------- */
/* Replaces PortOperatorBandDTBC (src/magnelio/ports/_modal/band_dtbc.py:
 * 780-1236) with its BandDTBCBoundary (:509-680).  Flat indices are into
 * the reference E (H) vectors; matrices row-major.  The port plane is
 * written from the p boundary coordinates (e[e_u] = Wu xt, e[e_v] = Wv xt),
 * the boundary couples to the first interior period through
 * M_coup (p x n1) and to the exterior through D0, Dm1 (p x p) and the
 * matrix DTBC kernels; the recorder projects n_modes channels: V with
 * me (n_u + n_v) and v_profile (n_modes x (n_u + n_v)) on the port plane
 * (u part plus v part), I with mh (n_h) and h_profile (n_modes x n_h) on
 * its dual faces, both times record_scale.  x1_prev0 may be NULL (a
 * quiescent start).  p <= 32, n_modes <= 16; before the first step; the
 * in-place stencil modes only (FITB_ERR_STATE in the fused forms). */
typedef struct {
    int32_t p, n_modes, n_kernel_init;
    int64_t n_u, n_v, n1, n_h;
    const int64_t *e_u_idx, *e_v_idx, *x1_idx, *h_idx;
    const double *Wu, *Wv, *M_coup, *D0, *Dm1;
    const double *me, *v_profile, *mh, *h_profile, *record_scale;
    const double* x1_prev0;
} fitb_band_desc;
int fitb_add_band_port(fitb_handle* h, const fitb_band_desc* d, int32_t* out_id);
/* Matrix DTBC kernel table L_m (m = 0..n_kernel-1, each p x p row-major) of
 * band port `port`, outgoing (incoming = 0) or incoming (1, excited ports):
 * lengths n0, 2 n0, 4 n0, ... in order, one call each; a step n uses the
 * table of the smallest length >= n + 1 (band_dtbc.py:591-603). */
int fitb_set_band_kernel(fitb_handle* h, int32_t port, int32_t incoming, int32_t n_kernel, const double* L);
/* Ghost source of field set b: n_samples p-vectors s^n (n_samples x p),
 * zero beyond (the synthesised series of set_excitation /
 * set_excitation_band, :940-1118); needs the incoming kernel. */
int fitb_set_band_source(fitb_handle* h, int32_t port, int32_t b, int64_t n_samples, const double* s);

/* ---- 2-D port modes --------------------------------------------------- */
/* The numerical core of Numerical2DModeSolver._solve_te_tm
 * (src/magnelio/ports/_modal/numerical_2d.py:454-585) on the GPU of
 * `device`, in float64: the n_modes lowest eigenvalues above `threshold`
 * of K v = lambda M v (K: the 2-D curl-curl stiffness on the n free port
 * edges as CSR, M: their epsilon-mass diagonal) with eigenvectors
 * normalised to v^T M v = 1, eigvecs [n_modes][n].  Dense Householder
 * tridiagonalisation of M^-1/2 K M^-1/2, bisection on the Sturm sequence,
 * inverse iteration, back-transformation.  The sign of each vector is the
 * caller's.  n <= 16384, n_modes <= 64; needs no handle. */
int fitb_mode_solve(int32_t device, int64_t n, const int64_t* rowptr, const int64_t* col, const double* val,
                    const double* m_diag, int32_t n_modes, double threshold, double* eigvals, double* eigvecs);

/* The lowest eigenpairs of a large sparse symmetric positive semi-definite
 * matrix L (CSR, n x n, float64), orthogonal to n_null given orthonormal
 * null vectors (row-major n_null x n): eigenvalues ascending into eigvals,
 * orthonormal eigenvectors row-major into eigvecs (n_modes x n).
 * Chebyshev-filtered subspace iteration on the device (degree 100 filters
 * on [a, b], b the row-sum bound of L, a the block's largest Ritz value;
 * Gram-Schmidt with reorthogonalisation; Rayleigh-Ritz), converged when
 * every wanted residual |L x - theta x| is below tol b, or after 20
 * iterations without halving once below 1e-12 b; at most 400 iterations,
 * else FITB_ERR_LIMIT.  `residual` (the largest wanted residual over b) and
 * `iterations` may be null.  The port-mode problems of large port planes:
 * the TE face form and the TM problem of a hollow guide (the reference
 * solves them with shift-invert ARPACK, numerical_2d.py:497-544, :585-650).
 * n <= 2^26, n_modes <= 16, n_null <= 8; needs no handle. */
int fitb_sparse_eigs(int32_t device, int64_t n, const int64_t* rowptr, const int64_t* col, const double* val,
                     int32_t n_null, const double* null_vecs, int32_t n_modes, double tol, double* eigvals,
                     double* eigvecs, double* residual, int32_t* iterations);

/* ---- surface-impedance walls ---------------------------------------- */
/* One SIBC wall tag (solver/_sibc.py:88-264, hooks at fit_td.py:837-840 and
 * :909-914): n_faces flat indices into the reference H vector with their
 * geometry factor g = A / l_dual^2, and per Foster branch of the wall's
 * impedance fit k = (1 - b dt/2)/(1 + b dt/2), q = c b dt/(1 + b dt/2).
 * The instantaneous part g R_inst must already be folded into the H
 * coefficients (the reference folds it into M_sigma_m).  Each step stashes
 * h on the faces first, then, right after the H update and the mu-side ADE
 * and before the H-side CPML corrections, adds beta_H g sum_p
 * ((1 + k_p)/2) u_p (every wall in order, so a face two walls book takes
 * both terms in wall order) and advances u_p <- k_p u_p + q_p h_mid with
 * h_mid the mean of the stashed and the new h.  Blocks of one handle are
 * kept in the order added; before the first step; in-place stencil modes
 * only (FITB_ERR_STATE in the fused forms). */
int fitb_add_sibc_block(fitb_handle* h, int64_t n_faces, const int64_t* idx, const double* g, int32_t n_branches,
                        const double* k, const double* q);

/* ---- plane waves ---------------------------------------------------- */
/* Replaces PlaneWaveSource.attach / inject_E / inject_H (plane_wave.py:229,
 * :720-733; called from fit_td.py:964-967, :990-993). */
int fitb_add_plane_wave(fitb_handle* h, const fitb_plane_wave_desc* d, int32_t* out_id);
/* Amplitude factor of plane wave `id` for field set b (default 1). */
int fitb_set_plane_wave_scale(fitb_handle* h, int32_t id, int32_t b, double scale);

/* ---- monitors ------------------------------------------------------- */
int fitb_add_dft_monitor(fitb_handle* h, const fitb_dft_desc* d, int32_t* out_id);
/* Complex bins of monitor `mon`, field set b, component c (0..5), shape
 * (n_freq, ni, nj, nk); re / im arrays of that many doubles. */
int fitb_read_dft(fitb_handle* h, int32_t mon, int32_t b, int32_t comp,
                  double* re, double* im, size_t count);

/* ---- time stepping -------------------------------------------------- */
/* Advance all field sets by n_steps leapfrog steps (the body of the loop
 * at fit_td.py:950-1007), replaying captured CUDA graphs. */
int fitb_step(fitb_handle* h, int64_t n_steps);
/* Blocks until every issued step has finished, then checks the device
 * status word that the pipelined kernels' bounded waits set (an expired
 * wait is an error); the reference's loop is synchronous at every step. */
int fitb_sync(fitb_handle* h);
/* Non-blocking: *done = 1 when every step issued so far has finished on the
 * device (then also the fitb_sync checks ran), 0 while work is in flight.
 * No counterpart in the reference (its loop is synchronous); the serving
 * loop uses it to keep every resident handle busy. */
int fitb_query(fitb_handle* h, int32_t* done);
/* Self-check of the device-side timeout path (no counterpart in the
 * reference): one CTA waits, bounded, on an mbarrier that nothing completes,
 * the expired wait records the timeout status (FITB_STATUS_WAIT_TIMEOUT) the
 * pipelined kernels use, and the host reads it into *status; the handle
 * stays usable.  No fault is involved. */
#define FITB_STATUS_WAIT_TIMEOUT 3
int fitb_probe_wait_timeout(fitb_handle* h, int32_t* status);
/* fitb_step bracketed by CUDA events on the handle's stream; blocks until
 * the steps are done and returns their device time in milliseconds. */
int fitb_step_timed(fitb_handle* h, int64_t n_steps, double* ms);
/* Measurement helper: device time of n_iter back-to-back launches of the E
 * update alone and of the H update alone (ms per launch).  It advances the
 * fields like n_iter half steps each, so call it only after the run whose
 * results are wanted. */
int fitb_time_stencil(fitb_handle* h, int32_t n_iter, double* ms_e, double* ms_h);
/* Steps taken so far (the solver's step counter n, fit_td.py:950). */
int fitb_steps_done(fitb_handle* h, int64_t* out);
/* 0.5 * (sum M_eps e^2 + sum M_mu h^2), float64 accumulation
 * (fit_td.py:1014-1018). */
int fitb_energy(fitb_handle* h, int32_t b, double* out);
/* Stored energy of caller-owned device arrays, without any device
 * allocation.  No counterpart in the reference: it exists for callers that
 * cannot allocate device memory while they run (a fixed device-memory
 * budget, an embedding framework that owns every device byte, or a loop
 * that must not incur the synchronisation cudaMalloc/cudaFree may cause).
 * e / m_eps hold n_e and h / m_mu hold n_h elements of the field dtype
 * (precision 4 = float32, 8 = float64); out is one device double receiving
 * 0.5 * (sum m_eps e^2 + sum m_mu h^2).  Work is enqueued on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) of the current device.
 * The block partial sums live in a fixed 1 MiB device array inside this
 * library (held on every device that uses it until the process exits), so
 * at most 131072 * 4096 elements per (e, h) pair are accepted; larger
 * sizes return FITB_ERR_LIMIT.  The first call on a device looks the array
 * up (cudaGetSymbolAddress) and should come before any stream capture.
 * Calls share the array: calls whose work overlaps on the GPU race.  A CUDA
 * error still pending from earlier work on the calling thread makes the call
 * return FITB_ERR_CUDA without launching anything (the error is left for its
 * owner to read). */
int fitb_energy_noalloc(const void* e, const void* h, const void* m_eps, const void* m_mu,
                        int64_t n_e, int64_t n_h, int32_t precision, double* out, void* stream);
/* max |V| * record_scale over all modal ports of field set b since the last
 * poll, then reset (operator.py:1323-1334 poll_signal_absmax). */
int fitb_poll_signal_absmax(fitb_handle* h, int32_t b, double* out);
/* Recorded V/I per channel for steps [step0, step0 + n): channel order is
 * port registration order, modes within a port (lumped ports: one channel).
 * V and I are [n][n_channels] (reference: src/magnelio/ports/recorder.py
 * :216-285). */
int fitb_channel_count(fitb_handle* h, int32_t* out);
int fitb_read_vi(fitb_handle* h, int32_t b, int64_t step0, int64_t n,
                 double* V, double* I);
/* The same read, asynchronous: D2H copies of steps [step0, step0 + n) of
 * field set b into V / I (page-locked host memory for an overlapped copy)
 * queued behind the issued steps; the ticket's completion (fitb_wait_ticket)
 * means the values have landed.  Statuses of the steps are checked by the
 * next synchronising call (fitb_sync, fitb_query, fitb_read_*).  A host loop
 * can so read each step's results while the next step runs. */
int fitb_read_vi_async(fitb_handle* h, int32_t b, int64_t step0, int64_t n, double* V, double* I, int64_t* ticket);
int fitb_wait_ticket(fitb_handle* h, int64_t ticket);
/* Modal S-parameters of the recorded steps [0, steps_done), computed on the
 * device from the V/I records without reading them back (replaces the host
 * post-step compute_s_parameters, src/magnelio/post/modal_sparameters.py
 * :335-545, over Signal1D.at_frequencies, src/magnelio/signals/
 * signal_1d.py:59-97): per field set and channel the direct DFT
 * sum_n x_n exp(-2 pi j f n dt) of V and I at the nf frequencies f [Hz], I
 * advanced by exp(+j pi f dt) unless icot[c] (I sampled with V), the power
 * waves a = aV V + aI I, b = bV V + bI I with the caller's per-channel maps
 * ([nch][4][nf] complex as (re, im) pairs: aV, aI, bV, bI), and
 * S[f][c][b] = b_c / a_excited[b] (complex, (re, im) pairs) where
 * |a_excited| >= a_threshold * its peak over f, NaN elsewhere and for field
 * sets with excited[b] = -1.  A (optional, [nf][B] complex) receives
 * a_excited.  Float64 throughout. */
int fitb_s_params(fitb_handle* h, int32_t nf, const double* f, const double* maps, const int32_t* icot,
                  const int32_t* excited, double a_threshold, double* S, double* A);

/* ---- checkpoint ----------------------------------------------------- */
/* Byte size of the full evolving state (fields, psi, port and monitor
 * state, step count) and its export / import (fit_td.py:1264-1353). */
int fitb_state_size(fitb_handle* h, size_t* out);
int fitb_state_export(fitb_handle* h, void* buf, size_t len);
int fitb_state_import(fitb_handle* h, const void* buf, size_t len);

#ifdef __cplusplus
}
#endif
#endif /* FITB200_H */
