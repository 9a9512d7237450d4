/*
 * pned_gpu.h -- C ABI of the B200 (sm_100a) implementation of pNED's
 * matrix-free H.v and the Krylov loops built on it.
 *
 * The entry points replace the single-rank (lnp = 1) hot path of pNED's
 * Fortran code.  Each declaration cites the reference routine it stands in
 * for (paths relative to the pNED project root; S1/2 = S_one_half/Hybrid_TPS_*,
 * Sa = S_arbitrary/Hybrid_TPS9_*).
 *
 * Conventions kept from the reference:
 *   - complex numbers are two doubles (re, im), layout-compatible with
 *     Fortran complex(KIND(0d0)) and C double _Complex;
 *   - local matrices xlocal are [9][Q][Q] column-major per bond type,
 *     Q = q_spin^2: element (row = target pair state, col = current pair
 *     state, type t) at row + Q*col + Q*Q*(t-1), exactly the memory of the
 *     Fortran array xlocal_Ham(0:Q-1,0:Q-1,9);
 *   - the pair state of a bond (s1 < s2) is d(s2)*q + d(s1); digit (bit) j
 *     of the basis index is site j+1;
 *   - H.v accumulates v0 += X(target, current) v1(partner), i.e. H^T
 *     (S1/2 parallel.f90:358), and prdct = <v1|H v1>.
 *   - batched vectors are interleaved: element (state s, vector r) at s*R + r.
 *
 * Every function returns PNED_OK (0) or an error code; the message of the
 * last error of the calling thread is returned by pned_last_error().  No call
 * exits or stops the process.  Pointer arguments marked "host or device"
 * are interpreted according to the PNED_PTR_DEVICE flag of the call.
 */
#ifndef PNED_GPU_H
#define PNED_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PNED_ABI_VERSION 1

/* status codes */
#define PNED_OK 0
#define PNED_EINVAL 1      /* invalid argument or model                         */
#define PNED_ENOMEM 2      /* device allocation failed                          */
#define PNED_EBUDGET 3     /* request exceeds the HBM budget of the context     */
#define PNED_EBREAKDOWN 4  /* Lanczos beta below 0.5e-30 (S1/2 Lanczos.f90:126) */
#define PNED_ECUDA 5       /* CUDA runtime error                                */
#define PNED_ETIMEOUT 6    /* a bounded wait gave up                            */
#define PNED_ENOTSUP 7     /* combination not supported by this build           */

/* pointer-location flags */
#define PNED_PTR_HOST 0
#define PNED_PTR_DEVICE 1

typedef struct { double re, im; } pned_c128;

typedef struct pned_model pned_model;
typedef struct pned_ctx pned_ctx;

/* ------------------------------------------------------------------------ */
/* library                                                                   */
/* ------------------------------------------------------------------------ */
int pned_abi_version(void);
const char *pned_last_error(void);
/* CUDA device used by models/contexts created afterwards on this thread. */
int pned_set_device(int device);

/* ------------------------------------------------------------------------ */
/* host-side model input (replaces set_xlocal_Ham / change_to_TPS_hamiltonian) */
/* ------------------------------------------------------------------------ */

/*
 * Local two-site matrices from the 19 coupling slots of the reference
 * (order: J1 K1 I11 I12 J1p K1p J1pp K1pp I11p I12p I11pp I12pp J2 K2 I21 I22
 * J3 K3 ratio_l), for tree 0 (S1/2 params.f90:1388-1563, q must be 2) or
 * tree 1 (Sa params.f90:1412-1602, any q).  field (may be NULL) adds the
 * Zeeman term -h.S_i split over the `coord` nearest-neighbour bonds of each
 * site (an extension: the reference has no field).  Also writes the skip mask
 * llocal_Ham (1 = skipped) and parity_type (S1/2 params.f90:1565-1595,
 * Sa params.f90:1604-1655).
 */
int pned_build_xlocal(int q_spin, int tree, const double *couplings19, int simple, const double *field3,
                      double coord, pned_c128 *xlocal_out, uint8_t *skip_out, int *parity_type_out);

/*
 * TPS Hamiltonian.  mode 0 reproduces change_to_TPS_hamiltonian
 * (S1/2 params.f90:1600-1623, Sa params.f90:1660-1686) and returns its L in
 * *L_inout; mode 1 uses the L given in *L_inout: X <- (L/n_bonds) 1 - X.
 */
int pned_tps_transform(int q_spin, int tree, int n_bonds, double c_count, int mode, pned_c128 *xlocal_inout,
                       double *L_inout);

/* Sz-sector basis list and Lin tables (S1/2 parallel.f90:452-578, Sa :366-486).
   With list1 == NULL only the dimension is returned in *ldim. */
int pned_mk_list12(int n_sites, int q_spin, int parity_type, int total_sz, int64_t *ldim, int64_t *list1,
                   int64_t *list3_lo, int64_t *list3_hi);

/* ------------------------------------------------------------------------ */
/* model                                                                     */
/* ------------------------------------------------------------------------ */
typedef struct {
    int32_t n_sites;          /* n                                                 */
    int32_t q_spin;           /* 2S+1                                              */
    int32_t tree;             /* 0: S1/2 schedule order, 1: Sa schedule order      */
    int32_t n_bonds;          /* ibond                                             */
    const int32_t *ipair;     /* [2*n_bonds] 1-based sites (ipair)                 */
    const int32_t *bond_type; /* [n_bonds] 1..9 (ibond_type)                       */
    const pned_c128 *xlocal;  /* [9][Q][Q] (xlocal_Ham)                            */
    const uint8_t *skip;      /* [9][Q][Q] llocal_Ham, 1 = skipped; NULL = none    */
    int32_t parity_type;      /* 0 = Sz-conserving sector basis, else full basis   */
    int32_t total_sz;         /* digit sum of the sector when parity_type == 0     */
} pned_model_desc;

/*
 * Compiles the bond table into the device term program (flip masks or
 * mixed-radix offsets with coefficient tables) and uploads it to the current
 * device.  Replaces set_parallel_bits + make_cpu_list2 + mk_list12
 * (S1/2 MPIlib.f90:74-84, 104-341; parallel.f90:452-578) for one GPU.
 * parity_type == 0 selects the Sz-conserving sector of digit sum total_sz
 * (mk_list12 order; vectors have the sector dimension, index = the
 * reference's list1 order); its diagonal must be real.
 */
int pned_model_create(const pned_model_desc *desc, pned_model **out);
int pned_model_destroy(pned_model *m);
/* dim = q^n; n_terms = off-diagonal gather terms per state in the program. */
int pned_model_info(const pned_model *m, int64_t *dim, int *n_terms, int *real_coefficients);
/*
 * Measurement hook (no counterpart in the reference): the H.v plan for R
 * vectors.  tile_passes = launches of the tiled kernel per H.v (0: the flat
 * gather kernel runs, or R > 1 not planned yet); partner_tiles = distinct
 * out-of-tile flip patterns summed over the passes (each one a partner-tile
 * read); tile_states = states per tile.  Any output may be NULL.
 */
int pned_model_plan(const pned_model *m, int R, int *tile_passes, int *partner_tiles, int *tile_states);
/*
 * Tuning hook (no counterpart in the reference): parameters of the tiled H.v
 * plan for R vectors; any field -1 keeps its default.  row_fixed_bits: low
 * global bits kept in the tile rows (8 for R = 1 by default: rows are runs
 * of 256 consecutive states; fewer lets the planner pick tile bits that
 * leave fewer partner tiles); window_bits: outer bits whose partner tiles a
 * pass expects in L2; max_passes: 1..4; j_bits (R = 1 only): 1..4, states
 * per thread 2^j_bits (fewer: fewer registers, more resident blocks; 4: tiles
 * of 4096 states, more flips inside the tile).  Re-plans at
 * once; call it between launches, not while other threads launch on the
 * model.  Used by the autotuner (pned_b200.tune).  plan NULL (and a model
 * whose plan was never set) takes the size's default: for R = 1 from 26
 * sites on, row_fixed_bits 5, window_bits 7, two passes, objective 1, stage
 * 3, two terms in flight (the plan the autotuner picks on B200 at 26-30
 * sites); otherwise every field at its own default as described here.
 */
typedef struct {
    int32_t row_fixed_bits;
    int32_t window_bits;
    int32_t max_passes;
    int32_t j_bits;
    int32_t l1_carveout;   /* 1 (default): shared-memory carveout sized to the tiles, the rest L1; 0: driver's choice */
    int32_t stage_partner_tiles; /* R = 1, j_bits 3: 1 copies each partner tile into shared memory once
                                    (cp.async); 2 streams own and partner tiles with bulk copies (TMA engine)
                                    through a ring of 32 KB shared-memory stages, one block per SM; 2 needs
                                    tile rows that keep >= 3 low global bits, else the plan uses 0; 3 gathers
                                    the partners as 0 and brings the tile's own rows, epilogue rows and
                                    diagonal in with tensor copies (TMA, no multicast); 3 needs every pass's
                                    tile bits (starting at bit 0) in at most 5 copy dimensions and two
                                    blocks per SM, else the plan uses 0 */
    int32_t blocks_per_sm; /* R = 1, j_bits 3: 3 builds the gather kernel for three resident blocks per SM
                              (85 registers, faster up to about 2^26 states); else two (the default) */
    int32_t objective;     /* how a pass picks its tile bits: 0 (default) the fewest partner tiles; 1 the
                              most flip terms inside the tile (each then gathers from shared memory instead
                              of through L1/L2) and window bits that take the most terms into the pass */
    int32_t terms_in_flight; /* stage 3: the partner rows of 2 out-of-tile terms requested together
                                (126 registers); else (0, 1, -1: default) one term at a time */
} pned_tile_plan;
int pned_model_set_plan(pned_model *m, int R, const pned_tile_plan *plan);
/*
 * Test and measurement hook (no counterpart in the reference): the tile plan
 * (S = 1/2 full basis) that the planner builds for this model with row_bits row
 * bits a tile (8: the single-vector kernel, as pned_model_set_plan; fewer: the
 * multi-vector kernel's 256 / G rows), computed on the host without device
 * work; the default fixed row bits are min(row_bits, 8), and plan NULL with
 * row_bits 8 gives the model's default plan (from 26 sites on fixed 5, window
 * 7, 2 passes, objective 1).  out[0..cap)
 * receives int64 values, *len the full count: the number of flip terms X, X
 * records (xmask, pos4, tab, nb), the number of passes, and per pass (tbits, jb,
 * nouter, nterms, nin, ngroups), rowpos[tbits], jpos[jb], outer[nouter], nterms
 * records (mask, pos4, jtab, tab, nb, hasj, lmask), gstart[ngroups + 1],
 * gxor[ngroups].  In-tile terms (the first nin) carry the local xor (row bits
 * 0..tbits-1, then the j bits), the others the global xor.
 */
int pned_tile_plan_export(const pned_model_desc *d, int row_bits, const pned_tile_plan *plan, int64_t *out,
                          int64_t cap, int64_t *len);
/*
 * Test hook (no counterpart in the reference): the mixed-radix tile passes of k
 * sites (q > 2, full basis; the `low` lowest sites in every tile) that the tiled
 * mixed-radix kernel runs, computed on the host.  out[0..cap) receives int64
 * values, *len the full count: q, n, the number of radix terms X, X records
 * (offset, s1, s2, tab), the table size T and T flags (entry nonzero), the
 * number of passes, and per pass (k, nouter, nterms), sites[k], outer[nouter],
 * nterms records (loff, ls1, ls2, tab).
 */
int pned_qtile_plan_export(const pned_model_desc *d, int k, int low, int64_t *out, int64_t cap, int64_t *len);
/*
 * Measurement hook (no counterpart in the reference): the partner-tile
 * staging the single-vector plan actually runs (0 gathered through L1/L2,
 * 1 cp.async, 2 bulk copies) and, for 2, the number of ring stages.
 */
int pned_model_tile_staging(const pned_model *m, int *mode, int *ring_stages);
/*
 * Measurement hook (no counterpart in the reference): S = 1/2 Sz-sector models
 * run the one-vector H.v per segment (the contiguous states sharing their high
 * half; one block per segment, partner ranks from one table read, high-half
 * flips rank for rank) when the largest segment has at least 256 states;
 * enable = 0 selects the flat gather with two Lin-table reads per term
 * instead, 1 the segment kernel again, -1 leaves the setting.  *active (may be
 * NULL) = 1 when the segment kernel runs.  Both give the same W bit for bit.
 */
int pned_model_sector_segments(pned_model *m, int enable, int *active);

/* ------------------------------------------------------------------------ */
/* context: device vectors for R interleaved vectors                         */
/* ------------------------------------------------------------------------ */
/* hbm_budget = 0: no budget check beyond the device's free memory. */
int pned_ctx_create(pned_model *m, int R, size_t hbm_budget, pned_ctx **out);
int pned_ctx_destroy(pned_ctx *c);
/* cudaStream_t used by the context (NULL = the context's own stream). */
int pned_ctx_set_stream(pned_ctx *c, void *stream);
int pned_ctx_synchronize(pned_ctx *c);
/* Device pointer of the context's interleaved vector buffer k (0..3). */
int pned_ctx_buffer(pned_ctx *c, int k, pned_c128 **dev_ptr);
/* Bytes of device memory the context holds. */
int pned_ctx_bytes(const pned_ctx *c, size_t *bytes);

/* ------------------------------------------------------------------------ */
/* vector kernels                                                            */
/* ------------------------------------------------------------------------ */

/*
 * p_mltply_v3 (S1/2 parallel.f90:190-263, Sa parallel.f90:184-261):
 * v0 += (H - eperbd*n_bonds)^T v1 for each of the R interleaved vectors, and
 * prdct[r] = <v1_r|(H - eperbd*n_bonds)^T v1_r>.  v1, v0 host or device
 * ([dim][R]); prdct host, may be NULL.
 */
int pned_hv(pned_ctx *c, const pned_c128 *v1, pned_c128 *v0, double eperbd, pned_c128 *prdct, int ptr_flags);

/*
 * Allocation-free H.v (no counterpart in the reference): the same product as
 * pned_hv on device vectors, v0 += (H - eperbd*n_bonds)^T v1 and
 * prdct[r] = <v1_r|...>, without a context and without allocating device
 * memory.  For callers that cannot call cudaMalloc: a host that hands all of
 * its HBM to its own pool (or to the resident state vectors) and would see a
 * hidden allocation fail or fragment that pool, or a thread that must not
 * allocate at all.  The reduction scratch is a fixed device array inside the
 * library (4096 complex values, 64 KB, held by every GPU that loads the
 * library until exit); R may be 1, 2, 3, 4, 6, 8, 12 or 16, and anything else
 * is rejected with PNED_EINVAL.  The first call on a device resolves the
 * array's device address (set-up).  The address is kept for the life of the process: after a
 * cudaDeviceReset of that device it is stale, so do not call this again on a
 * device that was reset.  Every call shares the array: calls that overlap on the GPU race and
 * must be ordered by the caller (one stream, or events).  v1, v0 are device
 * pointers ([dim][R]); prdct is host memory (may be NULL); stream is a
 * cudaStream_t (NULL = default stream); the call returns after the stream has
 * finished the product.
 */
int pned_hv_noalloc(const pned_model *m, int R, const pned_c128 *v1_dev, pned_c128 *v0_dev, double eperbd,
                    pned_c128 *prdct, void *stream);

/* calc_vec_inprdct (S1/2 parallel.f90:104-126): out[r] = sum conj(x1_r) x2_r. */
int pned_inprdct(pned_ctx *c, const pned_c128 *x1, const pned_c128 *x2, pned_c128 *out, int ptr_flags);

/* calc_beta (S1/2 parallel.f90:161-188): out[r] = sum |v0_r - alpha_r v1_r|^2. */
int pned_calc_beta(pned_ctx *c, const pned_c128 *alpha, const pned_c128 *v1, const pned_c128 *v0, double *out,
                   int ptr_flags);

/*
 * Seeded complex-Gaussian vectors (replaces the compiler-RNG initial vector of
 * parallelized_set_initial_vec_p, S1/2 parallel.f90:17-102): element g =
 * s*R + r is sqrt(-ln u1) e^{2 pi i u2} from splitmix64 counters; each vector
 * is then normalised when normalise != 0.  v_dev is a device pointer.
 */
int pned_fill_gaussian(pned_ctx *c, uint64_t seed, int normalise, pned_c128 *v_dev);

/* ------------------------------------------------------------------------ */
/* Krylov drivers                                                            */
/* ------------------------------------------------------------------------ */

/*
 * Lanczos (parallelized_lnc1z, S1/2 Lanczos.f90:48-163) on R independent
 * chains: n_steps values alpha[i*R + r], beta[i*R + r] (i = 0 .. n_steps-1,
 * the reference's alpha(i+1), beta(i+1)).  v_init ([dim][R], host or
 * device) must be normalised.  check_conv != 0 applies the nvec = 8
 * convergence stop of :133-155 (R = 1 only); *steps_done returns the number of
 * steps.  ene (may be NULL) receives the 8 lowest Ritz values of chain 0
 * (bisec, S1/2 basic.f90:25-107).
 */
int pned_lanczos_run(pned_ctx *c, const pned_c128 *v_init, int n_steps, int check_conv, double *alpha, double *beta,
                     double *ene, int *steps_done, int ptr_flags);

/*
 * Diagonal two-bit observable for the TPS step (S1/2 TPS.f90:128-321):
 * O(s) = sum_t c_t T[bit(s,a_t)][bit(s,b_t)], bit(s,p) = 0 for p >= n.
 */
typedef struct {
    int32_t n_terms;
    const int32_t *a;   /* [n_terms] bit positions */
    const int32_t *b;   /* [n_terms] bit positions */
    const pned_c128 *c; /* [n_terms] weights        */
    pned_c128 T[4];     /* T[2*i + k]               */
} pned_observable;

/*
 * mTPQ / TPS (parallelized_TPSz, S1/2 TPS.f90:325-409) on R interleaved seeds
 * with a model already transformed to L - H (pned_tps_transform).  Per step i
 * and seed r: alpha[i*R+r] = L - <k|(L-H)|k>, beta[i*R+r] = ||(L-H)|k>||,
 * coef[(i*R + r)*ncoef + j] with j = 0..4 as coef(i,1..5) of eval_phys_val
 * (:83-111) and 2 entries per observable.  ncoef = 5 + 2*n_obs.
 */
int pned_tps_run(pned_ctx *c, double L, const pned_c128 *v_init, int n_steps, int n_obs, const pned_observable *obs,
                 double *alpha, double *beta, double *coef, int ptr_flags);

/*
 * Dynamical structure factor chains (intalv_zz + parallelized_dsflnc1z,
 * S1/2 DSF.f90:18-87, 195-261; Sa DSF.f90:18-89): for r = 0..R-1 the start
 * vector is S^z_q x with phases qr[r*n + j] = q_r.r_j, normalised; cnorm[r] =
 * ||S^z_q x||^2 / n (sbeta(1)).  salpha[i*R + r] (i < n_steps) and
 * sbeta[i*R + r] (i <= n_steps, sbeta[0] = cnorm) as the reference's
 * salpha(i+1), sbeta(i+1).  x is one vector [dim] (host or device).
 */
int pned_dsf_run(pned_ctx *c, const pned_c128 *x, const double *qr, int n_steps, double *cnorm, double *salpha,
                 double *sbeta, int ptr_flags);
/*
 * The same chains started from S^{ipm}_q x (intalv_xy: the 'xx' component of
 * S1/2 DSF.f90:91-193, ipm = +1, bit j 0 -> 1; the 'uu'/'dd' components of Sa
 * DSF.f90:91-286, ipm = +1 / -1, digit d -> d + ipm with the spin-ladder factor
 * sqrt((S -+ m)(S +- m + 1))).  x lives on `source`'s basis (for a sector model
 * its states in mk_list12 order, the reference's listt), the chains on the
 * context's model (the target sector, Lin tables list3(:,:,0)); n and q must
 * match.  cnorm, salpha, sbeta as pned_dsf_run.
 */
int pned_dsf_xy_run(pned_ctx *c, const pned_model *source, int ipm, const pned_c128 *x, const double *qr, int n_steps,
                    double *cnorm, double *salpha, double *sbeta, int ptr_flags);

/*
 * parallelized_lncv1z (S1/2 Lanczos.f90:183-329), R = 1: replays the Lanczos
 * chain of v_init (host or device, as in pned_lanczos_run) with the stored
 * alpha/beta of the first pass and returns x = sum_k coef[k] v_k (coef[0..n_steps-1],
 * the tridiagonal eigenvector from pned_vec12) normalised, in x_out (host or
 * device).  As written the reference zeroes v1 before its first product, so
 * its x is the normalised initial vector, refined afterwards by inverse
 * iteration (pned_cg_run); this computes the Lanczos eigenvector the routine
 * sets up.
 */
int pned_lanczos_vector(pned_ctx *c, const pned_c128 *v_init, int n_steps, const double *alpha, const double *beta,
                        const double *coef, pned_c128 *x_out, int ptr_flags);
/*
 * Inverse iteration with CG (parallelized_inv1z + parallelized_cg1,
 * S1/2 cg.f90:18-196) for chain 0: b_init (normalised, [dim]) and E;
 * x_out receives the normalised eigenvector ([dim], host or device).
 */
int pned_cg_run(pned_ctx *c, double E, const pned_c128 *b_init, int inv_max, int cg_max, pned_c128 *x_out,
                int *n_inv, int *n_cg, int ptr_flags);

/* ------------------------------------------------------------------------ */
/* Krylov sessions: the same loops, advanced step by step on the device      */
/* ------------------------------------------------------------------------ */
/*
 * A session keeps the Krylov vectors of R chains resident in the context and
 * advances them in place, so a caller (a serving loop, a benchmark) can run
 * steps incrementally without host round trips.  pned_lanczos_run,
 * pned_tps_run and pned_dsf_run are begin + step + read + end.
 *
 * kind PNED_SESSION_LANCZOS: parallelized_lnc1z steps (S1/2 Lanczos.f90:97-157)
 *      from v_init; PNED_SESSION_TPS: parallelized_TPSz steps (S1/2
 *      TPS.f90:368-404) with total shift L (model already L - H) and optional
 *      observables; PNED_SESSION_DSF: parallelized_dsflnc1z chains
 *      (S1/2 DSF.f90:195-261) started from S^z_q x (pned_session_begin_dsf).
 */
#define PNED_SESSION_LANCZOS 1
#define PNED_SESSION_TPS 2
#define PNED_SESSION_DSF 3

int pned_session_begin(pned_ctx *c, int kind, const pned_c128 *v_init, int max_steps, double L, int n_obs,
                       const pned_observable *obs, int ptr_flags);
/* DSF chains: start vectors S^z_q x (intalv_zz, S1/2 DSF.f90:18-87); cnorm[r] = sbeta(1). */
int pned_session_begin_dsf(pned_ctx *c, const pned_c128 *x, const double *qr, int max_steps, double *cnorm,
                           int ptr_flags);
/* DSF chains started from S^{ipm}_q x with x on the source model's basis (see pned_dsf_xy_run). */
int pned_session_begin_dsf_xy(pned_ctx *c, const pned_model *source, int ipm, const pned_c128 *x, const double *qr,
                              int max_steps, double *cnorm, int ptr_flags);
/* Enqueues n_steps steps on the context's stream and returns without waiting. */
int pned_session_step(pned_ctx *c, int n_steps);
/*
 * Waits for the enqueued steps and copies the per-step results of all steps so
 * far: alpha/beta [steps][R] and, for TPS, coef [steps][R][ncoef] (any may be
 * NULL).  status_out (may be NULL) is 1 if a Lanczos beta fell below 0.5e-30.
 */
int pned_session_read(pned_ctx *c, double *alpha, double *beta, double *coef, int *steps_done, int *status_out);
/* Device pointer of the current Krylov vector C and its scale (v = scale * C). */
int pned_session_vector(pned_ctx *c, pned_c128 **dev_ptr, double *scale_out);
int pned_session_end(pned_ctx *c);
/*
 * Measurement hook (no counterpart in the reference): runs n_steps further
 * session steps one at a time with CUDA events on the context's stream around
 * the H.v kernel and around the whole step; returns their mean durations.
 */
int pned_session_profile(pned_ctx *c, int n_steps, double *hv_ms, double *step_ms);
/*
 * Checkpoint / restart of a session (the role of interval_dump /
 * interval_dump_read, S1/2 output.f90:50-211: a long run stops and resumes
 * later).  save waits for the session's steps and writes its state -- kind,
 * steps done, device scalars, alpha/beta (and TPS coefficients) so far, and
 * its three vectors -- to `path` (sections framed by 8-byte lengths).  load
 * starts the same session on a context of the same basis and R from such a
 * file, with room for max_steps steps in all (at least the saved count);
 * steps taken after a load continue the saved run exactly.  Sessions with
 * observables are not checkpointed (PNED_ENOTSUP).
 */
int pned_session_save(pned_ctx *c, const char *path);
int pned_session_load(pned_ctx *c, const char *path, int max_steps);
/* The context's session: kind (0 = none), steps enqueued, max_steps, TPS coefficients per step. */
int pned_session_info(const pned_ctx *c, int *kind, int *steps_done, int *max_steps, int *n_coef);
/*
 * A Lanczos session (R = 1) in the reference's checkpoint terms: the state
 * parallelized_lnc1z holds at the top of its next iteration (S1/2 Lanczos.f90:
 * 97-122), where interval_dump writes it (vec1 = v0, vec2 = v1; pned_write_
 * interval_dump).  After k >= 1 steps: w_out = v0 = H v_k - beta_{k-1} v_{k-1}
 * (the last product, before its alpha is taken off), v_out = v1 = v_k (the
 * normalised vector whose alpha is alpha[k-1]); dim states each, host or
 * device memory per flags (PNED_PTR_DEVICE).  Waits for the session's steps.
 */
int pned_session_lanczos_state(pned_ctx *c, pned_c128 *w_out, pned_c128 *v_out, int flags);
/* A DSF chain session (R = 1) has the same state in parallelized_dsflnc1z's terms
 * (S1/2 DSF.f90:234-257; its interval_dump passes vec1 = v1, vec2 = v0, sa = salpha,
 * sb = sbeta with sbeta(1) = cnorm): pned_session_lanczos_state exports it and
 * pned_session_begin_dsf_at resumes it (alpha = salpha[0..k-1], beta = sbeta[1..k]). */
int pned_session_begin_dsf_at(pned_ctx *c, const pned_c128 *w, const pned_c128 *v, const double *alpha,
                              const double *beta, int k, int max_steps, int flags);
/*
 * Starts a Lanczos session (R = 1) from that state, as interval_dump_read
 * resumes parallelized_lnc1z (:87-93): k >= 1 steps done, alpha[0..k-1],
 * beta[0..k-1] (host arrays; beta[k-1] > 0), w = v0 and v = v1 above (host or
 * device memory per flags); room for max_steps steps in all.  The next step forms (v0 - alpha[k-1] v1) / beta[k-1] and
 * continues the chain.
 */
int pned_session_begin_lanczos_at(pned_ctx *c, const pned_c128 *w, const pned_c128 *v, const double *alpha,
                                  const double *beta, int k, int max_steps, int flags);
/*
 * The same for a TPS session (R = 1, model built for L - H), in the terms of
 * parallelized_TPSz (S1/2 TPS.f90:366-395), whose interval_dump passes vec1 =
 * v0, vec2 = v1, vec3 = vg: after k >= 1 steps w_out = v0 = (L - H) v_k (not
 * normalised), v_out = v1 = v_k, g_out = vg = v_{k-1} (zero after one step).
 * begin_tps_at resumes from w and v (vg is overwritten by the loop's first
 * assignment), alpha/beta and the first five coefficient columns per step
 * (coef [k][5]: 2i/alpha1, L, beta, L - alpha1, <k-1|H|k>; a session without
 * observables).
 */
int pned_session_tps_state(pned_ctx *c, pned_c128 *w_out, pned_c128 *v_out, pned_c128 *g_out, int flags);
int pned_session_begin_tps_at(pned_ctx *c, double L, const pned_c128 *w, const pned_c128 *v, const double *alpha,
                              const double *beta, const double *coef, int k, int max_steps, int flags);

/* ------------------------------------------------------------------------ */
/* slot batches: continuous batching of chains with different couplings      */
/* ------------------------------------------------------------------------ */
/*
 * No counterpart in the reference, whose solvers run one chain per process;
 * each slot runs the reference's own recurrences:
 *   PNED_SLOT_LANCZOS  parallelized_lnc1z (S1/2 Lanczos.f90:48-163); also the
 *                      DSF momentum chains (parallelized_dsflnc1z, S1/2
 *                      DSF.f90:195-261) when loaded by pned_slots_load_szq
 *   PNED_SLOT_TPS      parallelized_TPSz with L - H (S1/2 TPS.f90:325-409),
 *                      coefficients as eval_phys_val (S1/2 TPS.f90:83-111)
 *   PNED_SLOT_VECTOR   parallelized_lncv1z (S1/2 Lanczos.f90:183-329): replays
 *                      a chain with its stored alpha/beta, x = sum_k c_k v_k
 * A batch holds R slots (R one of 1, 2, 3, 4, 6, 8, 12, 16) over one S = 1/2
 * lattice, fixed at creation by `structure` (sites, bonds, tree; its
 * couplings only fix which spin flips exist, so give it generic non-zero
 * local matrices).  Each slot carries its own couplings (same lattice,
 * real diagonal).  Vectors are the columns of interleaved [dim][R] buffers;
 * all slots advance together, one batched H.V per step, and slots are loaded
 * and released between steps while the others keep running.  Start vectors
 * are normalised on load.  Device memory: 16 dim R (3 vectors) + 8 dim R
 * (diagonals); hbm_budget (0: none) bounds it (PNED_EBUDGET).
 */
typedef struct pned_slots pned_slots;
#define PNED_SLOT_FREE 0
#define PNED_SLOT_LANCZOS 1
#define PNED_SLOT_TPS 2
#define PNED_SLOT_VECTOR 3

int pned_slots_create(const pned_model_desc *structure, int R, int max_steps, size_t hbm_budget, pned_slots **out);
int pned_slots_destroy(pned_slots *s);
int pned_slots_info(const pned_slots *s, int64_t *dim, int *R, int *max_steps, size_t *bytes);
/* stream: a cudaStream_t, or NULL for the batch's own stream */
int pned_slots_set_stream(pned_slots *s, void *stream);
/* kind PNED_SLOT_LANCZOS or PNED_SLOT_TPS (L: total shift of L - H); v_init [dim] */
int pned_slots_load(pned_slots *s, int slot, int kind, const pned_model_desc *couplings, const pned_c128 *v_init,
                    int n_steps, double L, int ptr_flags);
/* DSF momentum chain from S^z_q x (intalv_zz, S1/2 DSF.f90:18-87); qr [n] phases q.r_j */
int pned_slots_load_szq(pned_slots *s, int slot, const pned_model_desc *couplings, const pned_c128 *x,
                        const double *qr, int n_steps, int ptr_flags);
/* eigenvector pass: alpha/beta/coef [n_steps] of the first pass; x_dev [dim] device memory, overwritten */
int pned_slots_load_vector(pned_slots *s, int slot, const pned_model_desc *couplings, const pned_c128 *v_init,
                           int n_steps, const double *alpha, const double *beta, const double *coef,
                           pned_c128 *x_dev, int ptr_flags);
/* marks the slot free (its column keeps running as zeros) */
int pned_slots_release(pned_slots *s, int slot);
/* enqueues n_steps batch steps on the batch's stream and returns without waiting */
int pned_slots_step(pned_slots *s, int n_steps);
/* 1 when all enqueued work has finished, 0 while it runs, else an error status */
int pned_slots_query(pned_slots *s);
int pned_slots_synchronize(pned_slots *s);
/*
 * Waits for the batch's stream and reads one slot: kind, steps done, status
 * (1: beta breakdown), alpha/beta [steps_done] (TPS: L - alpha1 and beta),
 * TPS coef [steps_done][5] (2k/alpha1, L, beta, L - alpha1, Re(L<k-1|k> -
 * <k-1|L-H|k>)) and the DSF norm ||S^z_q x||^2 / (n ||x||^2).  Any output may
 * be NULL.
 */
int pned_slots_read(pned_slots *s, int slot, int *kind, int *steps_done, int *status, double *alpha, double *beta,
                    double *coef, double *cnorm);
/* Tuning and measurement hooks of the batch's tiled H.V (see pned_model_set_plan / pned_model_plan). */
int pned_slots_set_plan(pned_slots *s, const pned_tile_plan *plan);
int pned_slots_plan(const pned_slots *s, int *tile_passes, int *partner_tiles, int *tile_states);
/*
 * Column r of the seeded complex Gaussian [dim][R] start vectors of
 * pned_fill_gaussian (unnormalised), written as a dense [dim] device vector
 * on `stream` (a cudaStream_t, NULL: the default stream); returns without
 * waiting.  Replaces parallelized_set_initial_vec_p (S1/2 parallel.f90:17-102)
 * for one vector of a batch.
 */
int pned_gaussian_column(int64_t dim, int R, int r, uint64_t seed, pned_c128 *v_dev, void *stream);

/* ------------------------------------------------------------------------ */
/* host tridiagonal / continued-fraction routines                             */
/* ------------------------------------------------------------------------ */
/* bisec (S1/2 basic.f90:25-107) */
int pned_bisec(const double *alpha, const double *beta, int ndim, double *E, int ne, double eps);
/* vec12 (S1/2 basic.f90:112-213); v is [nvec][ndim] */
int pned_vec12(const double *alpha, const double *beta, const double *E, int ndim, int nvec, double *v);
/* exec_renbun (S1/2 DSF.f90:263-334): salpha/sbeta of length s_maxitr (zero padded) */
int pned_exec_renbun(int i_range, int s_maxitr, double split, double ene, double epsln, const double *salpha,
                     const double *sbeta, double *w, int *conv, double *dsf);
/* nomalization_DSF (S1/2 DSF.f90:337-351) */
int pned_normalize_dsf(int i_range, double split, double sq_re, double *dsf);

/* ------------------------------------------------------------------------ */
/* output chain of mTPQ runs                                                 */
/* ------------------------------------------------------------------------ */
/*
 * The TPQ coefficient file SalphaSbeta_me%05dseed%05d<comp> (dump_alpha_beta_coef,
 * S1/2 TPS.f90:507-538): Fortran unformatted sequential, five records --
 * num_data1 (int32), num_data2 (int32), alpha[num_data1], beta[num_data1],
 * coef[num_data2][num_data1] (column-major coef(k, m)) -- each framed by its
 * 4-byte length.  The reader returns the sizes; with alpha, beta and coef
 * non-NULL (capacity1 >= num_data1, coef room for num_data1 * num_data2)
 * it also fills them.
 */
int pned_write_salphasbeta(const char *path, int num_data1, int num_data2, const double *alpha, const double *beta,
                           const double *coef);
int pned_read_salphasbeta(const char *path, int *num_data1, int *num_data2, double *alpha, double *beta,
                          double *coef, int capacity1);
/*
 * eval_mpi (S1/2 eval_mpi.f90:236-363, 395-440): canonical averages of n_seeds
 * mTPQ runs on num_div + 1 temperatures log-spaced in [t_min, t_max].  Per
 * seed s (arrays [n_seeds][num_data1]): beta = the TPS norms, energy =
 * coef(:,4) = L - alpha1, hmix = coef(:,5) = Re<k-1|H|k>.  out[num_div+1][5]:
 * T, E(T) (seed mean), C(T) = dE/dT by the centred difference at
 * T +- t_delta (t_delta = 1e-4, or 0.9 t_min below that), the seed variance
 * of E averaged over T +- t_delta, and d2E/dT2.
 */
int pned_tpq_thermo(int num_data1, int n_seeds, const double *beta, const double *energy, const double *hmix,
                    double t_min, double t_max, int num_div, double *out);
/*
 * The ground-state vector file basisme%05d (readwrite_vec_data, S1/2
 * output.f90:12-36): two records, the energy e (double) and x[ll] (complex).
 * Records longer than one subrecord (2^31 - 9 bytes: ll > 134217727, every
 * vector from N = 27 on) are written and read as gfortran writes them: split
 * into subrecords, each framed by 4-byte length markers, the leading marker
 * negative when another subrecord follows and the trailing one negative when
 * one precedes.
 */
int pned_write_vec_data(const char *path, double e, const pned_c128 *x, int64_t ll);
int pned_read_vec_data(const char *path, double *e, pned_c128 *x, int64_t ll);
/* SalphaSbeta_q%05dme%05d<comp> (dump_alpha_beta, S1/2 DSF.f90:353-379): sq, salpha[s_maxitr], sbeta[s_maxitr]. */
int pned_write_dsf_alpha_beta(const char *path, pned_c128 sq, const double *salpha, const double *sbeta, int s_maxitr);
int pned_read_dsf_alpha_beta(const char *path, pned_c128 *sq, double *salpha, double *sbeta, int s_maxitr);
/* Appends one momentum's block of the text spectrum (write_dsf_res, S1/2 output.f90:246-264). */
int pned_append_dsf_res(const char *path, double sq_re, const double *q2, const double *w, const double *dsf,
                        const int *conv, int ll);
/* Appends the DSF driver's sq.txt line for momentum iq (S1/2 DSF.f90:490-492; Sa DSF.f90:578-580):
 * ' q = ', iq, q(1), q(2), Re sq in '(A,I3,2F12.6,F25.18)'. */
int pned_append_sq(const char *path, int iq, double q1, double q2, double norm_re);
/* vec_q%05dme%05d<comp> (dump_alpha_beta / read_alpha_beta2, S1/2 DSF.f90:374-379, 399-405):
 * records indx (int32), v1 [ll], v2 [ll]; long records in subrecords as pned_write_vec_data. */
int pned_write_dsf_vectors(const char *path, int indx, const pned_c128 *v1, const pned_c128 *v2, int64_t ll);
int pned_read_dsf_vectors(const char *path, int *indx, pned_c128 *v1, pned_c128 *v2, int64_t ll);
/*
 * The reference's checkpoint of a long run (interval_dump / interval_dump_read /
 * check_interval_dump, S1/2 output.f90:50-211; files DUMP_NAME = vecdump_me%05d
 * and DUMP_NAME.info).  The .info file holds one record each of DUMP_NAME
 * (character(128), blank padded), lnp, progress(7) (logicals, 4 bytes, 1 =
 * .true.), max_itr, dsf_comp (character(2)), s_maxitr, n, ibond, nvec,
 * total_sz, then itr_counter(1..12) one record each.  The data file holds
 * data_size, vec_size (int32 records), then the arrays the calling loop
 * passes, in this order and only those present: sa, sb, sc (column-major),
 * se (doubles), vec0, vec1, vec2, vec3, vec4 (data_size complex states each;
 * vec1 and vec2 always).  Long records are split into subrecords as
 * pned_write_vec_data does.  parallelized_lnc1z passes sa = alpha, sb = beta
 * (itr_counter(2) each), sc = coef (itr_counter(2) x 9), se = ene (max_itr),
 * vec1 = v0, vec2 = v1 (pned_session_lanczos_state).
 */
typedef struct {
    char dump_name[128];       /* DUMP_NAME as stored: blank padded, no terminator needed */
    int32_t np;                /* lnp, the run's MPI ranks */
    int32_t position[7];       /* progress(1..7): 0 or 1 */
    int32_t max_itr;
    char dsf_comp[2];
    int32_t s_maxitr, n, ibond, nvec, total_sz;
    int32_t itr_counter[12];
} pned_dump_info;
typedef struct {
    int32_t data_size;         /* states of each vector */
    int32_t vec_size;          /* length of the iteration arrays (itr_counter(2) or (12)) */
    double *sa, *sb, *sc, *se; /* null: not in the file */
    int64_t n_sa, n_sb, n_sc, n_se;
    pned_c128 *vec[5];         /* vec0 .. vec4; null: not in the file (vec1, vec2 required) */
} pned_dump_data;
/* Writes `path` and `path`.info. */
int pned_write_interval_dump(const char *path, const pned_dump_info *info, const pned_dump_data *d);
/* Reads `path`.info. */
int pned_read_interval_dump_info(const char *path, pned_dump_info *info);
/* Byte lengths of the data file's records (*count of them; the first `cap` into bytes). */
int pned_interval_dump_records(const char *path, int64_t *bytes, int cap, int *count);
/* Reads the data file into the arrays present in d (their lengths must match the
 * records; vectors data_size states); sets d->data_size and d->vec_size. */
int pned_read_interval_dump(const char *path, pned_dump_data *d);
/*
 * Largest payload of one subrecord for the writers above (no counterpart in the
 * reference; gfortran's -fmax-subrecord-length): 1 .. 2147483639 bytes, default
 * 2147483639.  The readers accept any subrecord split.  Process-wide.
 */
int pned_set_max_subrecord(int64_t bytes);

#ifdef __cplusplus
}
#endif
#endif /* PNED_GPU_H */
