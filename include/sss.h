/*
 * sss.h — C ABI of libsss.so, the B200 (sm_100a) N-body physics library.
 *
 * Every entry point takes plain pointers and sizes. Unless stated otherwise a
 * pointer argument is a DEVICE pointer owned by the caller (for example the
 * data_ptr() of a torch tensor); the library owns only the scratch memory that
 * lives inside an sss_ctx. Calls are asynchronous on the caller's stream
 * (`stream` is a cudaStream_t passed as void*, NULL = legacy default stream)
 * unless their comment says they synchronise.
 *
 * Errors: every int-returning call returns SSS_OK (0) or one of the SSS_ERR_*
 * codes; sss_last_error() gives the message of the last failing call on that
 * context. Kernels whose waits are bounded record SSS_ERR_TIMEOUT in a device
 * status word that sss_device_status() reads back.
 *
 * Threading: one sss_ctx per session; a context is not thread-safe.
 *
 * Reference interfaces each group replaces are cited as file:line within the
 * reference project (Peuqui/SolarSystemSimulator, directory backend/).
 */
#ifndef SSS_H
#define SSS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SSS_ABI_VERSION 1

/* status codes */
#define SSS_OK                    0
#define SSS_ERR_ARG               1  /* bad argument (shape, range, NULL)        */
#define SSS_ERR_TOO_MANY_MASSIVE  2  /* more than SSS_M_MAX massive bodies       */
#define SSS_ERR_GUARD             3  /* a step-count guard ran out               */
#define SSS_ERR_TIMEOUT           4  /* a bounded device wait gave up            */
#define SSS_ERR_CUDA              5  /* a CUDA runtime / cuFFT call failed       */
#define SSS_ERR_CAPACITY          6  /* an output buffer was too small           */

/* precision of the pair interaction in the all-pairs kernels */
#define SSS_PREC_F64    0   /* every operation in f64 (the drop-in path)          */
#define SSS_PREC_MIXED  1   /* f32 pair arithmetic on f64-differenced positions,
                               f32 partial sums folded into f64 accumulators      */

/* integrators of sss_selfgrav_step_batch */
#define SSS_INT_KDK       0 /* kick-drift-kick leapfrog (selfgrav_kernel.py:333-386) */
#define SSS_INT_YOSHIDA4  1 /* 4th-order Yoshida: KDK substeps w1, w0, w1           */

typedef struct sss_ctx sss_ctx;

/* ---------------------------------------------------------------- context */

/* ABI version of the loaded library (== SSS_ABI_VERSION of its header). */
int sss_abi_version(void);

/* Create a context bound to CUDA device `device`. */
int sss_create(int device, sss_ctx** out);

/* Free the context and its scratch. NULL is accepted. */
void sss_destroy(sss_ctx* ctx);

/* Message of the last failing call on ctx (never NULL). */
const char* sss_last_error(const sss_ctx* ctx);

/* Synchronise `stream`, then read and clear the device status word that
 * bounded waits write. Returns SSS_OK or the recorded SSS_ERR_* code. */
int sss_device_status(sss_ctx* ctx, void* stream);

/* Number of streaming multiprocessors of the context's device. */
int sss_num_sms(const sss_ctx* ctx);

/* ------------------------------------------------- all-pairs self-gravity
 *
 * Replaces `beschleunigung` (selfgrav_kernel.py:222-260):
 *   a_t = sum_s Gm_s (r_s - r_t) / (|r_s - r_t|^2 + eps2)^(3/2)
 * Body records are double4 {x, y, z, Gm} (z ignored when dim == 2; Gm is the
 * source's G*mass and is ignored for targets). Output acc4 is double4
 * {ax, ay, az, 0}. The self term contributes exactly 0 (zero offset).
 * Sources are summed in ascending index order inside each source chunk; the
 * chunk partials are added in ascending chunk order, so a result depends only
 * on the inputs and on (n_src, n_tgt, number of SMs), never on scheduling.
 * All pointers are device pointers with 16-byte alignment.
 */
int sss_allpairs_accel(sss_ctx* ctx, int dim, int precision,
                       const double* src4, int64_t n_src,
                       const double* tgt4, int64_t n_tgt,
                       double* acc4, double eps2, void* stream);

/* Plummer potential at the targets, phi_t = -sum_s Gm_s / sqrt(|d|^2+eps2),
 * in f64; the self term (zero offset) IS included (-Gm_t/eps), as in the
 * reference energy (test_selfgrav.py:54-63) before its diagonal correction.
 * Output phi is double [n_tgt]. */
int sss_allpairs_potential(sss_ctx* ctx, int dim,
                           const double* src4, int64_t n_src,
                           const double* tgt4, int64_t n_tgt,
                           double* phi, double eps2, void* stream);

/* Resident self-gravity state (caller-owned device buffers). Bodies
 * [0, n_src) are the massive sources, [n_src, n_src + n_tracer) massless
 * tracers (Kernel B, selfgrav_kernel.py:262-420). pos4[cur] holds the current
 * positions; the other buffer is the ping-pong target of each drift, and
 * `cur` is updated by every call that moves the bodies. acc4 holds the
 * accelerations at pos4[cur] once sss_selfgrav_init_accel has run. */
typedef struct sss_selfgrav_state {
    int      dim;         /* 2 or 3                                        */
    int      precision;   /* SSS_PREC_F64 or SSS_PREC_MIXED                */
    int64_t  n_src;       /* massive bodies (sources and targets)          */
    int64_t  n_tracer;    /* massless tracers (targets only)               */
    double*  pos4[2];     /* [n_src + n_tracer] {x, y, z, Gm}              */
    double*  vel4;        /* [n_src + n_tracer] {vx, vy, vz, 0}            */
    double*  acc4;        /* [n_src + n_tracer] {ax, ay, az, 0}            */
    int      cur;         /* 0 or 1: which pos4 buffer is current          */
    double   eps2;        /* Plummer softening squared, > 0                */
} sss_selfgrav_state;

/* Accelerations of all bodies at pos4[cur] into acc4. */
int sss_selfgrav_init_accel(sss_ctx* ctx, sss_selfgrav_state* st, void* stream);

/* `steps` integrator steps over the whole state (one launch sequence on
 * `stream`). Replaces the step loop of selfgrav_kernel (selfgrav_kernel.py:
 * 333-419) and NBodySelfGrav.step_batch (:558-627). Each force evaluation is
 * one kernel whose epilogue applies the closing half kick, writes the
 * snapshot and applies the next opening half kick and drift. If `snap` is
 * not NULL it is a device float buffer of steps rows; row s is
 * [x|y|(z)|vx|vy|(vz)] over the n_src sources followed by [x|y|(z)] over the
 * tracers, i.e. 2*dim*n_src + dim*n_tracer floats per row (the layout of
 * selfgrav_kernel.py:600-627 for dim == 2). Requires acc4 to be valid. */
int sss_selfgrav_step_batch(sss_ctx* ctx, sss_selfgrav_state* st,
                            int integrator, double dt, int steps,
                            float* snap, void* stream);

/* ------------------------------------------ few massive + many asteroids
 *
 * Replaces `frame_kernel` and the device side of NBodyCuda
 * (nbody_kernel.py:97-560, 617-1060): massive bodies (M <= SSS_M_MAX) act on
 * each other and on the asteroids, asteroids act back on the massive bodies,
 * asteroid x asteroid is ignored; 4th-order Yoshida with hierarchical
 * substeps and a private adaptive loop for close-encounter ("hot")
 * asteroids. All arrays are caller-owned device buffers: per dimension c the
 * asteroid arrays have n_ast entries and the massive arrays M entries
 * (dimension 2 needs only the first two pointers of each triple). */
#define SSS_M_MAX            64   /* nbody_kernel.py:58 */
#define SSS_K_MAX            16   /* nbody_kernel.py:59 */
#define SSS_SUB_SAMPLES_MAX  32   /* nbody_kernel.py:71 */

typedef struct sss_frame_state {
    int      dim;                 /* 2 or 3 */
    int64_t  n_ast;
    int      M;
    double*  ast_x[3];            /* positions  [n_ast] */
    double*  ast_v[3];            /* velocities [n_ast] */
    double*  ast_acc[3];          /* work: accelerations [n_ast] */
    double*  ast_m;               /* masses [n_ast] (scatter mode 2 writes) */
    unsigned char* ast_vis;       /* 0 = frozen and force-free */
    double*  ast_r;               /* contact radii (0 = never touches) */
    int64_t* ast_idx;             /* original body index of each asteroid */
    unsigned char* ast_hot;       /* work [n_ast] */
    double*  mas_x[3];            /* [M] */
    double*  mas_v[3];
    double*  mas_m;
    unsigned char* mas_vis;
    double*  mas_r;
    int64_t* mas_idx;             /* original body index of each massive body */
    double   G;                   /* G_AU = 4 pi^2 in AU/yr/Msun */
    double   softening;           /* added to r^2 (SOFTENING = 1e-6 AU^2) */
    double   max_sub_dt;          /* MAX_SUB_DT_YEARS */
    int      max_sub_steps;       /* MAX_SUB_STEPS_PER_FRAME */
    double   w1, w0;              /* Yoshida weights */
    int      massless_asteroids;  /* 1: every asteroid mass is 0 (no back-reaction) */
} sss_frame_state;

/* One launch of k raster samples of length dt_raster (frame_kernel). snap is
 * [k][2*dim][n_ast + M] floats in original body order ([x|y|(z)|vx|vy|(vz)],
 * the layout NBodyCuda.step_batch returns); sub_pos [k][m_sub][dim][n_ast]
 * and sub_n [k][n_ast] hold the hot asteroids' sub-samples (sub_n == m_sub:
 * gap-free); hit_t/hit_m [n_ast] the first contact time since the launch
 * start (< 0: none, the caller sets -1) and the compact massive index;
 * guard_used (device int) the number of substeps taken. */
int sss_frame_launch(sss_ctx* ctx, const sss_frame_state* st, double dt_raster, int k, int m_sub,
                     float* snap, float* sub_pos, unsigned char* sub_n, float* hit_t, int* hit_m,
                     int* guard_used, void* stream);

/* Point updates at compact slots (>= 0: asteroid, < 0: massive -slot-1) —
 * apply_updates (mode 0: set x,v), apply_deltas (mode 1: add to x,v; slots
 * must be unique), apply_body_state (mode 2: set x,v and mass)
 * (nbody_kernel.py:947-1010). vals is [m][2*dim] (mode 2: [m][2*dim+1]),
 * device memory. */
int sss_frame_scatter(sss_ctx* ctx, const sss_frame_state* st, const int64_t* slot,
                      const double* vals, int m, int mode, void* stream);

/* ------------------------------------------------------------ broadphase
 *
 * Asteroid x asteroid collision candidates on a uniform grid and their
 * exact tests — replaces `Erkennungskarte._hits` and `_zellschluessel`
 * (film_producer.py:223-321). Inputs are device arrays of n bodies (f32
 * snapshot x, y, vx, vy; f32 contact radii rr; u8 asteroid and visibility
 * flags); h is the cell size, halo the stripe halo, [lo, hi) the x stripe
 * this call owns (-inf/+inf for one card). The hit list is bit-exact against
 * the reference: out_hits receives up to `capacity` int32 triples
 * (offset index 0..4, a, b) in no particular order — sorted by (offset, a, b)
 * they are the reference's pairs (a, b) in its order. n_hits / n_cand (host)
 * receive the number of hits and of candidate pairs (the reference's
 * `kandidaten`). Synchronous. SSS_ERR_CAPACITY if more hits than capacity
 * were found (n_hits tells how many). */
int sss_broadphase(sss_ctx* ctx, const float* x, const float* y, const float* vx, const float* vy,
                   const float* rr, const unsigned char* is_ast, const unsigned char* vis, int64_t n,
                   double dt_y, double h, double halo, float lo, float hi, int* out_hits,
                   int64_t capacity, int64_t* n_hits, int64_t* n_cand, void* stream);

/* ------------------------------------------------------ particle mesh, 2-D
 *
 * The reference's isolated 2-D PM (pm_kernel.py:34-293): Hockney-James zero
 * padding to 2N x 2N, convolution with the transforms of the softened force
 * kernels, cloud-in-cell deposit and gather, f64. A plan object holds the
 * cuFFT plans and the grids of one grid size N. All pointers are device
 * pointers. */
typedef struct sss_pm2d sss_pm2d;
int  sss_pm2d_create(sss_ctx* ctx, int grid_n, sss_pm2d** out);
void sss_pm2d_destroy(sss_pm2d* p);
/* bbox4 <- (xmin, xmax, ymin, ymax) of n points (grid_fuer, pm_kernel.py:110-124) */
int  sss_pm2d_bbox(sss_pm2d* p, const double* x, const double* y, int64_t n, double* bbox4, void* stream);
/* transforms of K_x, K_y = -G d / (|d|^2 + eps2)^1.5 for cell size h (:34-60) */
int  sss_pm2d_build_kernels(sss_pm2d* p, double h, double eps2, double G, void* stream);
/* acceleration field of n masses on the grid with origin (x0, y0) (:127-147) */
int  sss_pm2d_field(sss_pm2d* p, const double* gx, const double* gy, const double* gm, int64_t n,
                    double x0, double y0, double h, void* stream);
/* field read back at n points with the deposit's stencil (:93-107, :150-154) */
int  sss_pm2d_gather(sss_pm2d* p, const double* px, const double* py, int64_t n, double x0, double y0,
                     double h, double* ax, double* ay, void* stream);
/* the N x N crops of the last field into ax, ay (the arrays pm_force_field returns) */
int  sss_pm2d_fields(sss_pm2d* p, double* ax, double* ay, void* stream);
/* the N x N density of the last field call into rho (:63-90) */
int  sss_pm2d_density(sss_pm2d* p, double* rho, void* stream);
/* KDK piece (:264-273): v += hdt a; if drift, x += dt v */
int  sss_pm2d_kick_drift(sss_pm2d* p, double* x, double* y, double* vx, double* vy, const double* ax,
                         const double* ay, int64_t n, double hdt, double dt, int drift, void* stream);
/* out[i] = (float)a[i] (snapshot rows, :274-280) */
int  sss_pm2d_to_f32(sss_pm2d* p, const double* a, int64_t n, float* out, void* stream);

/* ------------------------------------------------ batched small systems
 *
 * Many independent systems of <= 64 bodies, f64 Yoshida-4 with a fixed
 * per-system dt, `steps` steps in one persistent launch. Bodies of all
 * systems are concatenated (x[c], v[c], m; system s owns [off[s], off[s+1]));
 * G[s], dt[s] per system; the launch integrates the systems listed in
 * sys_list[0..n_list) (all with at most max_n bodies) with a team of `team`
 * lanes (1, 2, 4, 8, 16 or 32) holding `per_lane` bodies each
 * (team * per_lane >= max_n). blocks = 0 picks one team per system.
 * Pair force: the softened all-pairs formula within each system (eps2 may
 * be 0; the self pair is excluded). No reference counterpart: the reference
 * integrates one system at a time (nbody_kernel.py, index.html engines). */
int sss_batched_launch(sss_ctx* ctx, int dim, double* const* x, double* const* v, const double* m,
                       const int64_t* off, const double* G, const double* dt, const int* sys_list,
                       int n_list, int max_n, int team, int per_lane, double eps2, int steps, int blocks,
                       void* stream);

/* ----------------------------------------------- no-allocation variant
 *
 * sss_allpairs_accel_noalloc computes exactly what sss_allpairs_accel
 * computes, for callers that may not allocate device memory: a host
 * application that owns the whole device-memory budget and hands libraries
 * only the buffers it sized in advance (an engine with its own arena
 * allocator, a plugin host that forbids library allocations), or a
 * latency-critical loop that cannot afford cudaMalloc/cudaFree, which block
 * and synchronise the device. It needs no sss_ctx and calls no cudaMalloc,
 * cudaFree or allocating library routine.
 *
 * Its scratch is one file-scope device array of SSS_NOALLOC_SCRATCH_BYTES
 * that every GPU loading libsss holds until the process exits. Limits: in
 * mixed precision n_src <= SSS_NOALLOC_MAX_MIXED_SOURCES (the f32 source
 * tiles must fit), SSS_ERR_CAPACITY otherwise; f64 has no source limit.
 * When the chunk partial sums of the source split do not fit, the split is
 * narrowed (down to a single chunk), which changes only the order in which
 * chunk partials are added (rounding-level differences).
 *
 * The first call on a device does a one-time set-up with that device
 * current (it resolves the array's device address with
 * cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call shares the array and finds the previous call's contents in it;
 * the call clears what must start at zero. Calls whose work overlaps on the
 * GPU (different streams, or devices sharing no order) race on the array:
 * order them on one stream.
 *
 * device: CUDA device of all pointers (made current). d_status: optional
 * device int that a timed-out bounded wait sets to SSS_ERR_TIMEOUT (NULL =
 * an internal word). errbuf/errbuf_len: optional host buffer for a message.
 * No reference counterpart. */
#define SSS_NOALLOC_SCRATCH_BYTES     (32u << 20)
#define SSS_NOALLOC_MAX_MIXED_SOURCES 1044480
int sss_allpairs_accel_noalloc(int device, int dim, int precision,
                               const double* src4, int64_t n_src,
                               const double* tgt4, int64_t n_tgt,
                               double* acc4, double eps2, int* d_status,
                               void* stream, char* errbuf, size_t errbuf_len);

/* ------------------------------------------------------------ diagnostics */

/* Measured FMA throughput of the device in TFLOP/s (2 flops per FMA lane):
 * kind 0 = f64 DFMA, 1 = f32 FFMA, 2 = packed f32x2 FMA. Synchronous; the
 * roofline denominator of the all-pairs kernels. No reference counterpart. */
int sss_probe_fma(sss_ctx* ctx, int kind, int iters, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* SSS_H */
