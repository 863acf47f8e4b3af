/*
 * thistle_b200 -- C-ABI of the B200 scattering-intensity path.
 *
 * Drop-in for THISTLE's Fortran calculation dispatcher and integrators:
 * plain pointers and sizes, Fortran (column-major, 1-based index) layouts
 * where the reference uses them, no torch types.  Every entry returns 0 on
 * success or a negative THISTLE_ERR_* code and never exits the process;
 * thistle_last_error_string() describes the last failure of the calling
 * thread.  All computation runs on the current CUDA device; there is no CPU
 * fallback.
 */
#ifndef THISTLE_B200_H
#define THISTLE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define THISTLE_OK 0
#define THISTLE_ERR_ARG -1        /* null pointer or bad size */
#define THISTLE_ERR_SHAPE -2      /* inconsistent group / index layout */
#define THISTLE_ERR_ANGMOM -3     /* l, m or n above 4 (g), or LLmax beyond the Bessel tables */
#define THISTLE_ERR_NONFINITE -4  /* NaN or Inf in an input array */
#define THISTLE_ERR_CUDA -5       /* CUDA runtime or kernel failure */
#define THISTLE_ERR_NOMEM -6      /* device allocation failed */
#define THISTLE_ERR_TYPE -7       /* calculation type not provided */
#define THISTLE_ERR_Q -8          /* q <= 0 (the reference divides by q; drivers use 1e-10 for 0) */

/* Measured FP64 FMA throughput of the current device in TFLOP/s (a
 * register-resident chain kernel, best of `reps`); the roofline denominator. */
int thistle_probe_fp64_peak(int32_t reps, double *tflops);

/* Calculation types, numbered as src/main_calculation.f90:99-497. */
#define THISTLE_TOTAL_J0 1
#define THISTLE_ELASTIC_J0 2
#define THISTLE_TOTAL_ALIGNED 3
/* elastic aligned: |F(q)|^2 with F the Fourier transform of the electron
 * density (elastic_integration_alig, src/Integrals.f90:2366-2490; CASE(4),
 * src/main_calculation.f90:218-265); Entry 1 and thistle_plan_form_factor. */
#define THISTLE_ELASTIC_ALIGNED 4
#define THISTLE_TOTAL_J2 7
/* elastic j2: the P2-weighted orientational average of the elastic
 * intensity (elastic_integration_j2, src/Integrals.f90:1941-2365; dispatch
 * CASE(8), src/main_calculation.f90:407-419); needs the 1-RDM like type 2. */
#define THISTLE_ELASTIC_J2 8
/* energy-resolved CMS: the elastic j0 kernel on zi_ab zj_cd, zi and zj the
 * AO densities of two (transition) 1-RDMs, summed over every ordered pair of
 * group pairs with weights 4, 2, 2, 1 (resolved_cms_integration,
 * src/Integrals.f90:2598-2930; variables_resolved_cms, src/Variables.f90:
 * 1283-1410; CASE(9), src/main_calculation.f90:438-471 and :820-846).  onerdm
 * holds the two (nmo1, nmo1) matrices back to back: the bra's, then the
 * ket's.  Plans of this type have no batch or adjoint form. */
#define THISTLE_RESOLVED_CMS 9
/* total j1 (CASE(10), src/main_calculation.f90:473-497): the reference's
 * tot_integration_j1 prints and stops before integrating
 * (src/Integrals.f90:526-527), so no result exists to reproduce; Entry 1 and
 * thistle_plan_create return THISTLE_ERR_TYPE with that reason. */
#define THISTLE_TOTAL_J1 10
/* electron scattering: I_e - 2 Ine + Inn (src/main_calculation.f90:277-329,
 * 330-...), I_e the total (5) or elastic (6) j0 intensity, Ine the
 * nuclear-electron term, Inn the nuclear-nuclear sinc sum; Entry 1 only.
 * Needs Zn (natoms), geom (natoms x 3, column-major) and the 1-RDM; type 5
 * also the 2-RDM rows.  q_abs_out receives q. */
#define THISTLE_TOTAL_ELECTRON 5
#define THISTLE_ELASTIC_ELECTRON 6

const char *thistle_last_error_string(void);
int thistle_version(void);

/*
 * Entry 1.  Replaces main_calculation_mod::total_scattering_calculation_2 with
 * readrdm=.True. (src/main_calculation.f90:501-849; f2py call shape of
 * total_scattering_calculation, :13-15, as driven by
 * src/scattering_main_routine.py:240-247).  RDMs come in as arrays instead of
 * files: mat/total/nmat are read_twordm's rows (src/one_rdm.f90:2112-2147),
 * onerdm is read_onerdm's matrix (:2072-2108).
 *
 *   type          1 total j0, 2 elastic j0, 3 total aligned, 4 elastic
 *                 aligned, 5 / 6 electron, 7 total j2, 8 elastic j2,
 *                 9 resolved CMS (10, total j1, is refused as the reference
 *                 stops there)
 *   Zn, geom      atomic numbers and (natoms,3) geometry; not used by these
 *                 types (kept for the reference's argument list), may be NULL
 *   maxl          maxval(l) as the reference passes it (checked, not trusted)
 *   ga,l,m,n,xx,yy,zz  per primitive function, length ngto
 *   mmod          (norbs, ngto) column-major MO coefficients of the primitives
 *   q, nq         radial momentum transfer grid, q > 0
 *   group         1-based shell index per function; shells contiguous
 *   cutoffz, cutoffmd, cutoffcentre  the reference's three cutoffs
 *   mat, total, nmat   (nmat,4) column-major 1-based MO indices and values
 *                      (types 1 and 7)
 *   onerdm, nmo1  (nmo1,nmo1) column-major 1-RDM (types 2, 4, 6 and 8); two
 *                 of them back to back for type 9
 *   q_abs_out     nq doubles, set to q (the reference returns |q| here)
 *   result_out    nq doubles, I(q)
 * Type 4 (CASE(4), src/main_calculation.f90:218-265) evaluates the elastic
 * aligned intensity |F(q)|^2 on the reference's own grid of nq vectors
 * (thistle_elastic_aligned_grid); q is not read, q_abs_out gets |q|, and the
 * 1-RDM is needed as for type 2.
 * Type 3 (CASE(3), src/main_calculation.f90:156-217) evaluates the aligned
 * intensity on the reference's own QCOORD3 grid (k0 = 10.583544175): nq must
 * be 3131, q is not read, q_abs_out gets |q| of the grid vectors and
 * result_out the real part of I(q) (the reference writes it, with the
 * imaginary part, to result_aligned.dat; the imaginary part is zero, see
 * thistle_plan_execute_aligned).
 * All pointers are host pointers.
 */
int thistle_total_scattering(int32_t type, const double *Zn, const double *geom, int32_t natoms,
                             int32_t maxl, int32_t ngto, int32_t ng, const double *ga,
                             const int32_t *l, const int32_t *m, const int32_t *n,
                             const double *xx, const double *yy, const double *zz,
                             const double *mmod, int32_t norbs, const double *q, int32_t nq,
                             const int32_t *group, double cutoffz, double cutoffmd,
                             double cutoffcentre, const int32_t *mat, const double *total,
                             int32_t nmat, const double *onerdm, int32_t nmo1,
                             double *q_abs_out, double *result_out);

/*
 * Plan interface: one basis, density and q grid set up once (density
 * transform on the device), then executed for any number of geometries.
 * The routine-level split of variables_total / tot_integration
 * (src/Variables.f90:948-1153, src/Integrals.f90:8-472).
 */
typedef struct thistle_plan thistle_plan;

int thistle_plan_create(thistle_plan **plan, int32_t type, int32_t ngto, const double *ga,
                        const int32_t *l, const int32_t *m, const int32_t *n, const double *xx,
                        const double *yy, const double *zz, const int32_t *group,
                        const double *mmod, int32_t norbs, const int32_t *mat,
                        const double *total, int32_t nmat, const double *onerdm, int32_t nmo1,
                        const double *q, int32_t nq, double cutoffz, double cutoffmd,
                        double cutoffcentre);
/* Type THISTLE_TOTAL_ALIGNED plans take q as nq vectors, a (3, nq)
 * column-major array (the reference's q_al layout), and evaluate
 * tot_integration_aligned (src/Integrals.f90:1425-1573) on them;
 * thistle_plan_execute then returns the real part.  This returns both parts:
 * the reference sums all ng^4 ordered quartets, whose bra-ket exchange
 * conjugates each term, so the imaginary part is zero (written as 0.0; the
 * reference's own is rounding noise).  im_host may be NULL. */
int thistle_plan_execute_aligned(thistle_plan *plan, double *re_host, double *im_host);
/* Adjoint of total j0 (type 1) with respect to the Gaussian centres.  No
 * counterpart in the reference.  For a cotangent v (nq doubles) it returns
 * grad[3 g + axis] = sum_q v(q) dI(q)/dA_g,axis for every group g (ng x 3,
 * row-major): the centre of group g is A_g; a nuclear gradient is the sum over
 * the groups on that atom.  The pair density (MO coefficients and RDM) is held
 * fixed; McMurchie-Davidson coefficients, Gaussian-product prefactors and the
 * Bessel argument |P_kr - P_ij| carry the geometry.  Quartets on the P = Q
 * branch contribute through their prefactors and coefficients only (that
 * branch does not depend on H).  Runs the forward stages first unless the
 * last execution used the current centres.  LLmax <= 8 (s, p, d shells). */
int thistle_plan_vjp(thistle_plan *plan, const double *v_host, double *grad_host);
/* Same with device pointers, on the plan's stream (no synchronisation). */
int thistle_plan_vjp_device(thistle_plan *plan, const double *v_dev, double *grad_dev);
/*
 * Geometry batches (no reference counterpart; the reference evaluates one
 * geometry per call).  A plan can hold ngeom geometries of its basis that
 * share its density, quartet list and stage-2 visiting order; every kernel
 * then runs over all of them in one launch (the geometry is the grid's second
 * dimension).  set_batch replicates geometry 0's centres into all slots;
 * set_centres_batch takes ngeom x ngto x 3 interleaved host coordinates.
 * execute_batch returns ngeom x nq doubles, vjp_batch takes ngeom x nq
 * cotangents and returns ngeom x ng x 3 group-centre gradients (type 1).
 * The single-geometry entry points work on geometry 0 of a batch.
 * use_graph makes the batch entry points capture their launches once in a
 * CUDA graph (forward, and the adjoint stages) and replay it; the graph is
 * dropped when the batch size changes.
 * autotune_batch times forward + adjoint per geometry for ngeom = 1, 2, 4, ..
 * <= gmax and two stage-2 q tiles, then the four stage-2 pair tiles at the
 * best of those, keeps the fastest (ngeom, q tile, pair tile) in the plan
 * and reports it with its geometries per second (stage2_tile reads the pair
 * tile).  set_stage2_tile sets the pair tile: quartets per lane 1 or 2,
 * warps per block 4 or 8 (default 2 x 4); aligned plans have none.
 */
int thistle_plan_set_batch(thistle_plan *plan, int32_t ngeom);
int thistle_plan_set_centres_batch(thistle_plan *plan, const double *xyz);
int thistle_plan_execute_batch(thistle_plan *plan, double *result_host);
int thistle_plan_execute_batch_device(thistle_plan *plan, double *result_dev);
/* Centres of every geometry from device memory (ngeom x ngto x 3,
 * interleaved), copied on the plan's stream without synchronising; the
 * functions of a group must share their centre (not checked here, unlike
 * set_centres_batch). */
int thistle_plan_set_centres_batch_device(thistle_plan *plan, const double *xyz_dev);
int thistle_plan_vjp_batch(thistle_plan *plan, const double *v_host, double *grad_host);
int thistle_plan_vjp_batch_device(thistle_plan *plan, const double *v_dev, double *grad_dev);
int thistle_plan_use_graph(thistle_plan *plan, int32_t enable);
int thistle_plan_autotune_batch(thistle_plan *plan, int32_t gmax, int32_t *ngeom_best, int32_t *qtile_best,
                                double *geoms_per_s);
int thistle_plan_set_stage2_tile(thistle_plan *plan, int32_t quartets_per_lane, int32_t warps_per_block);
/* Stage overlap (default on): each LLmax class's stage-2 visiting order is
 * sorted right after its stage 1, and its stage 2 starts on the plan's
 * internal streams while the later classes' stage 1 runs.  Off: stage 2
 * starts after the whole of stage 1.  The result is the same either way. */
int thistle_plan_set_pipeline(thistle_plan *plan, int32_t enable);
int thistle_plan_stage2_tile(const thistle_plan *plan, int32_t *quartets_per_lane, int32_t *warps_per_block);
/*
 * Nuclear-electron term of an elastic plan (type 2) for its current centres:
 * ine_host[q] = sum_a Zn_a sum over ordered group pairs (i,k) of the pair's
 * Hermite expansion against the plan's AO density at H = R_a - P_ik, times
 * e12 (nuclei_electron_integration, src/Integrals.f90:2493-2596, with
 * integral_k_ij :6192-6326 and integral_ij_pzero :4865-4953).  geom is
 * (natoms, 3) column-major.  Entry 1 types 5 and 6 combine it as
 * I_e - 2 Ine + Inn.
 */
int thistle_plan_nuclear(thistle_plan *plan, const double *Zn, const double *geom, int32_t natoms,
                         double *ine_host);
/*
 * Elastic plans (types 2, 8): the Fourier transform of the electron density,
 * F(q) = sum over ordered group pairs of e12(|q|) e^{i q.P} sum Z E E E (i q)^tuv
 * (elastic_integration_alig with integral_k_ijkr_alig, src/Integrals.f90:
 * 2366-2490, 6085-6190), for the plan's current centres on nq q vectors
 * (qvec: (3, nq) column-major, host).  re/im get F, abs2 |F|^2 (the type 4
 * intensity); any of the three may be NULL.
 */
int thistle_plan_form_factor(thistle_plan *plan, const double *qvec, int32_t nq, double *re_host,
                             double *im_host, double *abs2_host);
/* The nq q vectors of CASE(4) (src/main_calculation.f90:227-241), written as
 * a (3, nq) column-major array.  Host-only. */
int thistle_elastic_aligned_grid(int32_t nq, double *q_al);

/*
 * Molecule batches (no reference counterpart).  Several plans -- any bases,
 * one geometry each, the same calculation type, nq <= 1024 -- executed
 * together: the pair tables and the reductions run as one launch over every
 * plan, stage 1 as one launch per kernel shape, and stage 2 as ONE
 * persistent launch whose resident blocks take (plan, class, block) work
 * items from an atomic counter, heaviest Bessel order first; each item
 * writes its own partial rows, so results do not depend on the schedule.
 * batch_create runs every plan once (records and stage-2 visiting order)
 * and builds the launch tables; the plans must outlive the batch and keep
 * their stream.  execute writes the plans' I(q) one after the other (sum of
 * their nq doubles).  use_graph captures the launches once in a CUDA graph
 * and replays it.  info: [0] plans, [1] total q points, [2] kernels
 * launched by the last execution.
 * set_stage2_tile picks the stage-2 pair tile (quartets per lane 1 or 2,
 * warps per block 4 or 8; default 2 x 4) and stage2_tile reads it; autotune
 * times the batch at the four tiles, keeps the fastest and reports it with
 * its molecules per second.  The plan functions of the same names do this
 * for one plan (thistle_plan_autotune_batch tunes the tile too).
 */
typedef struct thistle_batch thistle_batch;
int thistle_batch_create(thistle_batch **batch, thistle_plan *const *plans, int32_t nplans);
int thistle_batch_use_graph(thistle_batch *batch, int32_t enable);
int thistle_batch_execute(thistle_batch *batch, double *result_host);
int thistle_batch_execute_device(thistle_batch *batch, double *result_dev);
int thistle_batch_info(const thistle_batch *batch, int64_t *info);
int thistle_batch_set_stage2_tile(thistle_batch *batch, int32_t quartets_per_lane, int32_t warps_per_block);
int thistle_batch_stage2_tile(const thistle_batch *batch, int32_t *quartets_per_lane, int32_t *warps_per_block);
int thistle_batch_autotune(thistle_batch *batch, int32_t *quartets_per_lane, int32_t *warps_per_block,
                           double *molecules_per_s);
int thistle_batch_destroy(thistle_batch *batch);
/* The 3131 aligned q vectors of the reference (QCOORD3,
 * src/main_calculation.f90:864-929) for beam wavevector k0, written as a
 * (3, 3131) column-major array.  Host-only. */
int thistle_qcoord3(double k0, double *q_al);
/* Run the plan on a caller-owned cudaStream_t (passed as void*); the plan
 * stops using its own stream.  The caller keeps the stream alive. */
int thistle_plan_set_stream(thistle_plan *plan, void *stream);
/* Move the Gaussian centres (host arrays of length ngto). */
int thistle_plan_set_centres(thistle_plan *plan, const double *xx, const double *yy,
                             const double *zz);
/* Run the integrator for the current centres; result_host gets nq doubles. */
int thistle_plan_execute(thistle_plan *plan, double *result_host);
/* Same, leaving I(q) in device memory (nq doubles) on the plan's stream. */
int thistle_plan_execute_device(thistle_plan *plan, double *result_dev);
/* Redo the whole device pipeline from the device-resident inputs (density
 * transform, quartet enumeration, then the integrator); I(q) to device memory. */
int thistle_plan_recompute_device(thistle_plan *plan, double *result_dev);
/* Evaluate only the listed group quartets (0-based gi,gj,gk,gr, 4 int32 each,
 * each with its reference loop weight); result_host gets nq doubles. */
int thistle_plan_execute_quartets(thistle_plan *plan, const int32_t *quartets, int64_t nquart,
                                  double *result_host);
/* Counts: [0] group quartets, [1] LLmax classes, [2] ng, [3] ngto, [4] nq,
 * [5] kernels of this library launched by the last call. */
int thistle_plan_info(const thistle_plan *plan, int64_t *info6);
/* Per LLmax = 0..16: (LLmax, quartets, quartets on the P=Q branch in the
 * last execution) -- 51 int64 values. */
int thistle_plan_class_counts(const thistle_plan *plan, int64_t *out51);
/* Device time in ms: [0] pair tables, [1] stage 1, [2] stage 2 (Bessel sum),
 * [3] reduce of the last execution; [4] density transform and [5] quartet
 * enumeration of the set-up. */
int thistle_plan_timings(const thistle_plan *plan, double *ms6);
/* Waits for the plan's stream, then sums the device time of each stage
 * ([0] pair tables, [1] stage 1, [2] stage 2, [3] reduce) over the executions
 * since the previous call (at most the last 64); *nexec gets their number. */
int thistle_plan_stage_totals(thistle_plan *plan, double *ms4, int64_t *nexec);
/* The stage-1 records of the last execution and the q grid, in device memory
 * owned by the plan (valid until its next execution or destroy).  Per LLmax
 * class c < *ncls (at most 20 classes; the arrays need that room): quartets
 * [cls_begin[c], cls_end[c]) in class order, their records at cls_recoff[c]
 * doubles with stride cls_rs[c].  A record is [H, 1/4p+1/4p', kind (0 Bessel
 * j0, 1 Bessel j2, 2 P=Q polynomial in q^2), order, coefficients...].
 * Total, elastic and j2 plans only: aligned plans hold Hermite densities
 * instead and return THISTLE_ERR_TYPE. */
int thistle_plan_records(const thistle_plan *plan, const double **rec_dev, int32_t *ncls,
                         int64_t *cls_begin, int64_t *cls_end, int64_t *cls_recoff,
                         int32_t *cls_rs, const double **q_dev);
/* The plan's density after the MO -> primitive transform, copied to host
 * memory (no reference counterpart; for inspecting the transform).  Total
 * and j2 plans: the pair density rho, np x np with np = ngto (ngto + 1) / 2,
 * rho[P(a,b) np + P(c,d)] = ztot of functions a, b (electron 1) and c, d
 * (electron 2) -- zcontrred + zcontrred2 of src/Integrals.f90:109-127 and
 * 5163 -- with P(a,b) = max(a,b) (max(a,b) + 1) / 2 + min(a,b), 0-based.
 * Elastic plans: the AO density Z (ngto x ngto, column-major) of
 * variables_elastic (src/Variables.f90:1199-1217); resolved CMS plans: zi
 * then zj (2 ngto^2 doubles).  `count` is the capacity
 * of out in doubles; *needed receives the size either way (out may then be
 * NULL to query it). */
int thistle_plan_density(const thistle_plan *plan, double *out, int64_t count, int64_t *needed);
int thistle_plan_destroy(thistle_plan *plan);

/*
 * Device buffers released by plans stay cached in the library (per device) and
 * are reused by later plans of a similar size, so that repeated plans and
 * thistle_total_scattering calls do not pay cudaMalloc/cudaFree each time; a
 * failed allocation returns the cache to the driver and retries.  No
 * counterpart in the reference (whose arrays are Fortran allocatables).
 * thistle_release_device_cache frees the cached buffers and idle cuBLAS
 * handles of the current device; thistle_device_cache_bytes reports the bytes
 * cached and the bytes held by live plans on the current device.
 */
int thistle_release_device_cache(void);
int thistle_device_cache_bytes(int64_t *cached, int64_t *in_use);

/*
 * Stage 2 without any device allocation.  No counterpart in the reference
 * (whose integrators allocate freely on the host).  For callers that cannot
 * call cudaMalloc when they evaluate -- a host application that hands this
 * library device buffers and forbids allocations, or one that has already
 * given all device memory to its own pool -- this evaluates the Bessel sum of
 * stage-1 records the caller already holds (thistle_plan_records layout) on
 * the caller's q grid and writes nq doubles of I(q) to result_dev, on `stream`.
 * Its scratch is a fixed 2.4 MB array inside the library (296 blocks x 1024 q
 * points), so nq is limited to 1024 per call; larger nq is rejected with
 * THISTLE_ERR_ARG.  The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress) with the device current; make that first call
 * before any stream capture.  The address is kept for the life of the
 * process: a cudaDeviceReset (or anything else that destroys the device's
 * primary context) makes it stale, so do not call this entry point on a
 * device after resetting it.  All calls on a device share the array and it
 * keeps the last call's contents: calls that overlap on the GPU (different
 * streams, or threads) race and must be serialised by the caller.  The class
 * table must start at quartet 0 (cls_begin[0] == 0) and its ranges must be
 * contiguous; otherwise THISTLE_ERR_SHAPE.
 */
int thistle_bessel_sum_static(const double *rec_dev, int32_t ncls, const int64_t *cls_begin,
                              const int64_t *cls_end, const int64_t *cls_recoff,
                              const int32_t *cls_rs, const double *q_dev, int32_t nq,
                              double *result_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* THISTLE_B200_H */
