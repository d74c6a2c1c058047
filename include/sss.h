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
#define SSS_PREC_MIXED_TC 2 /* the same pair terms with the squared distances
                               formed on the tensor cores (split-TF32 products over
                               tile-centred f32 offsets), rsqrt and sums on the CUDA
                               cores, f32 tile sums folded into f64; tiles close to
                               a target block take the f32 pair loop. Needs
                               eps2 > 0.                                          */

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
    int      fine_guard;          /* iteration limit of a hot asteroid's fine loop
                                     (0 = SSS_FINE_GUARD, the reference's 8000) */
    int      pair_f32;            /* 1: asteroid x massive pair forces of calm asteroids
                                     and the back-reaction in f32 (offsets formed in f64,
                                     f32 rsqrt, sums in f64); hot asteroids' fine loops and
                                     massive x massive pairs stay f64. 0: all f64 */
} sss_frame_state;
#define SSS_FINE_GUARD 8000

/* One launch of k raster samples of length dt_raster (frame_kernel). When
 * the substep guard (max_sub_steps) or a fine-loop guard (fine_guard) runs
 * out before its interval is covered, the launch stops that interval there
 * as the reference does (nbody_kernel.py:248-250, :424) and records
 * SSS_ERR_GUARD in the device status word (sss_device_status). snap is
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
/* sort k hits of sss_broadphase in place into the reference's output order,
 * (offset, a, b) ascending: it concatenates one part per neighbour offset,
 * each ascending in (a, b) (film_producer.py:255-290); n = the bodies of the
 * call (a, b < n < 2^30) */
int sss_broadphase_order(sss_ctx* ctx, int* hits, int64_t k, int64_t n, void* stream);

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
/* one caller-held N x N f64 field (row stride ld >= N, device) read at n
 * points with the deposit's stencil; replaces _cic_gather (:93-107) */
int  sss_pm2d_gather_field(sss_ctx* ctx, const double* field, int grid_n, int64_t ld, const double* px,
                           const double* py, int64_t n, double x0, double y0, double h, double* out,
                           void* stream);
/* the N x N crops of the last field into ax, ay (the arrays pm_force_field returns) */
int  sss_pm2d_fields(sss_pm2d* p, double* ax, double* ay, void* stream);
/* the N x N density of the last field call into rho (:63-90) */
int  sss_pm2d_density(sss_pm2d* p, double* rho, void* stream);
/* KDK piece (:264-273): v += hdt a; if drift, x += dt v */
int  sss_pm2d_kick_drift(sss_pm2d* p, double* x, double* y, double* vx, double* vy, const double* ax,
                         const double* ay, int64_t n, double hdt, double dt, int drift, void* stream);
/* out[i] = (float)a[i] (snapshot rows, :274-280) */
int  sss_pm2d_to_f32(sss_pm2d* p, const double* a, int64_t n, float* out, void* stream);

/* ------------------------------------------------- collision response
 *
 * The per-sample collision analysis of the asteroid films (2-D), on the
 * device. Arrays are device arrays over the n bodies of a sample: f32
 * snapshot rows x, y, vx, vy; f32 contact radii rr; u8 visibility and
 * asteroid flags; f64 masses and radii. Both calls are synchronous (counts
 * return to the host).
 *
 * sss_collide_sweep replaces analyze_merge (film_producer.py:707-779): the
 * alive massive bodies m_idx[0..m_count) (vis and mass > 0) against every
 * alive body, the segment from the previous positions (px, py) to this
 * sample and the segment extrapolated by dt_y, in f32 as the reference;
 * pairs receives int32 triples (massive, body, fraction bits as f32) in the
 * reference's row-major order, runaways the bodies with v^2 > 9 v_esc^2
 * from the massive barycentre (ascending). SSS_ERR_CAPACITY when more than
 * cap_pairs / cap_run were found (the counts tell how many).
 *
 * sss_collide_bounce replaces bounce_deltas (:916-1019) for the broadphase
 * hits (sss_broadphase triples, any order; n <= SSS_COLLIDE_MAX_BODIES): hits
 * sorted into the reference's order, at most one hit per body (greedy in
 * that order), impulse with restitution e and overlap push in f64.
 * pairs_out receives the active hits as int32 (a, b) pairs in order
 * (capacity n_hits pairs); touched_out the bodies they touch, ascending
 * (capacity min(n, 2 n_hits)), deltas_out their (dx, dy, dvx, dvy). */
#define SSS_COLLIDE_MAX_BODIES 1600000
int sss_collide_sweep(sss_ctx* ctx, int64_t n, const float* gx, const float* gy, const float* gvx, const float* gvy,
                      const float* px, const float* py, const float* rr, const unsigned char* vis,
                      const unsigned char* is_ast, const double* mass, const int64_t* m_idx, int m_count,
                      double dt_y, double G, int* pairs, int64_t cap_pairs, int* runaways, int64_t cap_run,
                      int64_t* n_pairs, int64_t* n_run, void* stream);
int sss_collide_bounce(sss_ctx* ctx, int64_t n, const float* x, const float* y, const float* vx, const float* vy,
                       const double* real_r, const double* mass, const int* hits, int64_t n_hits, double dt_y,
                       double e, int* pairs_out, int64_t* touched_out, double* deltas_out, int64_t* n_act,
                       int64_t* n_touched, void* stream);
/* Fragmentation of fast asteroid x asteroid impacts (no counterpart in the
 * reference's producer, which only detects a body x body shatter at 1.5
 * v_esc, film_producer.py:801-822, and leaves the fragments to its client's
 * shatter(), index.html:7705-7745). For each of the n_pairs active bounce
 * pairs (int32 (a, b), e.g. sss_collide_bounce's pairs_out) in order whose
 * impact speed |v_b - v_a| >= factor * sqrt(2 G (m_a + m_b) / (r_a + r_b))
 * (and m_a + m_b > 0): parents_out receives (a, b) and frags_out n_frag
 * records (x, y, vx, vy, m, r) f64: equal masses, radii keeping the volume,
 * positions on a ring of radius r_a + r_b about the centre of mass,
 * velocities the centre's plus a scatter of speed v_imp (0.25 + 0.35 U) at
 * angle 2 pi k / n_frag + 0.6 (U - 1/2) with its mean removed (mass and
 * momentum conserved); U from SplitMix64 of (seed, a, b, k). factor 0 turns
 * it off. *n_events (host) receives the count; SSS_ERR_CAPACITY beyond cap.
 * Synchronous. */
int sss_collide_fragment(sss_ctx* ctx, int64_t n, const float* x, const float* y, const float* vx,
                         const float* vy, const double* real_r, const double* mass, const int* pairs,
                         int64_t n_pairs, double G, double factor, int n_frag, uint64_t seed, int* parents_out,
                         double* frags_out, int64_t cap, int64_t* n_events, void* stream);

/* ------------------------------------------------------- film ring slots
 *
 * sss_ring_slot replaces schreibe_slot (film_producer.py:79-123): one ring
 * slot (device bytes, slot_bytes = 8n + 4 + sub_max (4 + 8 m_sub)) from a
 * frame snapshot row (device f32 [x|y|...], at least 2n values) and the
 * sample's sub-samples as sss_frame_launch leaves them (sub_pos
 * [m_sub][dim][n_ast], sub_n [n_ast]; a_idx [n_ast] the original index of
 * every asteroid slot, ascending). Writes x|y, the count, the indices of the
 * hot asteroids (gap-free chains) ascending and their chains (nh, mSub, 2);
 * at most sub_max are kept (the lowest indices). *n_hot (host) receives how
 * many were hot (more than sub_max = overflow). Synchronous. Entries beyond
 * the count are left as they were.
 *
 * sss_ring_reorder replaces the self-gravity row reorder (:1245-1261): K rows
 * [x_m|y_m|vx_m|vy_m|x_t|y_t] (nm masses at original indices sg_m, nt tracers
 * at sg_t) into K rows [x|y|vx|vy] of n bodies in original order, tracer
 * velocities 0. */
int sss_ring_slot(sss_ctx* ctx, const float* row, int64_t n, const float* sub_pos, const unsigned char* sub_n,
                  const int64_t* a_idx, int64_t n_ast, int m_sub, int dim, int64_t sub_max, unsigned char* slot,
                  int64_t* n_hot, void* stream);
int sss_ring_reorder(sss_ctx* ctx, const float* rows, int K, const int64_t* sg_m, int64_t nm, const int64_t* sg_t,
                     int64_t nt, int64_t n, float* out, void* stream);

/* ------------------------------------------------------- stream frames
 *
 * The server's per-sample stream core (server.py: build_frame :378-537,
 * _anzeige_koords :99-111, _lod_auswahl :629-684, _dichte_filter :686-747,
 * _index_hash :117-131) on the device, with the reference's arithmetic.
 * sss_stream_sample: the bodies of one f32 sample (x, y) that are alive
 * (kill_t > t_cut) and inside box (host: x0, y0, spanx, spany as the
 * session's floats), thinned by the density LOD to about `budget` points
 * (massive bodies first, then the system's asteroids, then injected ones;
 * injected may be NULL), ascending in sel (u32), with their u16 box
 * coordinates; log_zoom uses the log-radial display coordinates. *n_sel
 * (host) receives the count; sel/qx/qy need capacity n. Synchronous.
 * sss_stream_minmax: (min x, max x, min y, max y) of the display coordinates
 * of all n bodies into out4 (host), the input of the automatic box. */
int sss_stream_sample(sss_ctx* ctx, int64_t n, const float* x, const float* y, const double* kill_t, double t_cut,
                      const unsigned char* is_ast, const unsigned char* injected, const double* box, int log_zoom,
                      int64_t budget, unsigned* sel, uint16_t* qx, uint16_t* qy, int64_t* n_sel, void* stream);
int sss_stream_minmax(sss_ctx* ctx, int64_t n, const float* x, const float* y, int log_zoom, float* out4,
                      void* stream);
/* Log-zoom display coordinates of n bodies (replaces _anzeige_koords with
 * log_zoom, server.py:99-111): q = p * log1p(r) / (log 33 * r), r = |p|, in
 * f32 with the C library's rounding of hypot and log1p; 0 where r <= 1e-9.
 * x, y, qx, qy are device arrays of n floats. Asynchronous. */
int sss_stream_display(sss_ctx* ctx, int64_t n, const float* x, const float* y, float* qx, float* qy,
                       void* stream);
/* sss_stream_sample_batch: k samples of the same bodies at once, as build_frame
 * packs the samples of one frame (server.py:378-537): x[i], y[i] (host arrays of
 * k device pointers) and t_cut[i] (host) per sample, the other inputs shared;
 * sample i's output at sel/qx/qy + i n (capacity k n each), its count in
 * n_sel[i] (host). One readback and one synchronisation for the batch. */
int sss_stream_sample_batch(sss_ctx* ctx, int64_t n, int k, const float* const* x, const float* const* y,
                            const double* kill_t, const double* t_cut, const unsigned char* is_ast,
                            const unsigned char* injected, const double* box, int log_zoom, int64_t budget,
                            unsigned* sel, uint16_t* qx, uint16_t* qy, int64_t* n_sel, void* stream);

/* ------------------------------------------------ particle mesh, 3-D periodic
 *
 * The reference's PM cycle (TODO.md:225-253; 2-D code pm_kernel.py:63-154)
 * in a periodic cube of side `box` on an n^3 f32 mesh: cloud-in-cell deposit
 * with warp-aggregated atomics, one R2C transform, one fused kernel for the
 * Green's function -4 pi G / k^2 * W(k)^-deconv * exp(-k^2 r_split^2)
 * (W the CIC window; deconv = 2 undoes deposit and interpolation, the
 * Gaussian is the long-range filter that keeps it from amplifying the
 * mesh-scale aliasing) and the spectral gradient -i k_d (the 1/n^3 of the
 * inverse folded in), one batched C2R for the three components, and
 * trilinear (CIC) interpolation into f64 accelerations. cuFFT performs only the transforms. A plan holds the
 * meshes and plans of one mesh size; particles stay with the caller.
 *
 * Particle state (device pointers, SoA f64): x[3], v[3], a[3]; masses m[n]
 * or, when m is NULL, every particle has mass_const. Positions are kept
 * wrapped into [0, box). */
typedef struct {
    int64_t n;
    double* x[3];
    double* v[3];
    double* a[3];
    const double* m;
    double mass_const;
} sss_pm3_particles;

/* epilogue of a force pass (the KDK pieces fused into the kernel that
 * produces the accelerations; v += hdt a is a half kick):
 * SSS_PM3_FORCE: a only; SSS_PM3_KICK: a, then v += hdt a;
 * SSS_PM3_KICK_DRIFT: a, v += hdt a, f32 snapshot row, v += hdt a,
 * x = wrap(x + dt v) (the closing kick of this step and the opening kick
 * and drift of the next). */
#define SSS_PM3_FORCE      0
#define SSS_PM3_KICK       1
#define SSS_PM3_KICK_DRIFT 2

typedef struct sss_pm3 sss_pm3;
int  sss_pm3_create(sss_ctx* ctx, int mesh_n, double box, sss_pm3** out);
void sss_pm3_destroy(sss_pm3* p);
/* internal meshes: rho (n^3 f32 density = mass / h^3) and the three
 * acceleration meshes (3 n^3 f32, contiguous), valid until the next call */
int  sss_pm3_meshes(sss_pm3* p, float** rho, float** accel);
/* deposit (rho) -> transforms -> acceleration meshes */
int  sss_pm3_density(sss_pm3* p, const sss_pm3_particles* s, void* stream);
int  sss_pm3_solve(sss_pm3* p, double G, int deconv, double r_split, void* stream);
/* interpolate the meshes at the particles into s->a and run the epilogue
 * `mode`; snap (nullable) receives the f32 row [x|y|z|vx|vy|vz] (6 n) */
int  sss_pm3_gather(sss_pm3* p, const sss_pm3_particles* s, int mode, double hdt, double dt, float* snap,
                    void* stream);
/* opening half kick and drift of one KDK step: v += hdt a; x = wrap(x + dt v) */
int  sss_pm3_kick_drift(sss_pm3* p, const sss_pm3_particles* s, double hdt, double dt, void* stream);
/* short-range part of a P3M force (no reference counterpart: the exact
 * complement of a mesh solved with r_split = 1 / (2 alpha)): adds
 * G m (erfc(alpha r) + 2 alpha r e^{-alpha^2 r^2} / sqrt(pi) + (1 + eps^2 /
 * r^2)^{-3/2} - 1) d / r^3 over the pairs closer than r_cut (nearest
 * periodic image, r_cut <= box / 3) to the accelerations in s->a (a mesh
 * force from an SSS_PM3_FORCE gather), then runs the epilogue `mode` as
 * sss_pm3_gather does */
int  sss_pm3_short(sss_pm3* p, const sss_pm3_particles* s, double G, double alpha, double r_cut, double eps,
                   int mode, double hdt, double dt, float* snap, void* stream);

/* ------------------------------------------------ Ewald direct sum, f64
 *
 * The judge of the mesh forces: the exact periodic force of point masses
 * with Plummer softening eps2 on the nearest image (Ewald summation,
 * Hernquist, Bouchet & Suto 1991): a real-space part over the nearest image
 * of every source within r_cut (r_cut <= box/2), and a reciprocal part over
 * the nk half-space vectors h (int32 triples, device) with per-vector
 * coefficient coef[k] = 2 * 4 pi / box^3 * exp(-|k|^2 / (4 alpha^2)) / |k|^2,
 * k = 2 pi h / box. No reference counterpart (the reference has no periodic
 * solver); it plays the role of its all-pairs check (test_selfgrav.py:66-88).
 *
 * sss_ewald_structure: sc[2k], sc[2k+1] <- sum_j m_j cos, sin(k . x_j);
 * hmax >= every |h| component of the list (<= 40; a vector outside it, or
 * with h_x < 0, contributes nothing).
 * sss_ewald_accel: accelerations at n_tgt target positions (t[3], device);
 * self_idx (nullable) names the source each target is (skipped). */
int sss_ewald_structure(sss_ctx* ctx, const sss_pm3_particles* src, double box, const int* hvec,
                        int nk, int hmax, double* sc, void* stream);
int sss_ewald_accel(sss_ctx* ctx, const sss_pm3_particles* src, const double* const* t,
                    const int64_t* self_idx, int64_t n_tgt, double G, double box, double alpha,
                    double r_cut, double eps2, const int* hvec, const double* coef, const double* sc,
                    int nk, double* const* out, void* stream);
/* sss_ewald_gtab: the host-built table of g(x) = erfc(x) + 2 x exp(-x^2) / sqrt(pi)
 * that the real-space sum evaluates (*n_int intervals of width *h over [0, n_int h],
 * 6 Taylor coefficients about each interval's centre, lowest order first) into
 * out (host, capacity cap doubles); host code only, no device call. */
int sss_ewald_gtab(double* out, int64_t cap, int* n_int, double* h);

/* ------------------------------------------- learned short-range correction
 *
 * A per-particle MLP 67 -> 128 -> 128 -> 3 (SiLU) that adds the short-range
 * force the mesh cannot resolve. Inputs: log1p(rho / rho_mean) on the 4x4x4
 * mesh cells around the particle's cell (i0-1 .. i0+2 per axis), then the
 * sub-cell offsets - 1/2 (padded with zeros to 80). Weights and activations
 * are bf16 on the tensor cores (tcgen05.mma, accumulators in tensor memory),
 * accumulation f32; forward, backward and the weight gradients all run
 * there. Parameters are one f32 array of SSS_MLP_N_PARAMS: W1[80][128],
 * b1[128], W2[128][128], b2[128], W3[128][8], b3[8] (rows 67..79 of W1 and
 * columns 3..7 of W3 zero); sss_mlp_pack turns them into the bf16 operand
 * images (SSS_MLP_N_FRAGS uint32: W1^T, W2^T and W2 in the tensor cores'
 * shared-memory layout, W3) that the kernels copy to shared memory. No
 * reference counterpart. */
#define SSS_MLP_N_PARAMS 27912
#define SSS_MLP_N_FRAGS  22016
#define SSS_MLP_IN_PAD   80
int sss_mlp_pack(sss_ctx* ctx, const float* params, uint32_t* frags, void* stream);
/* X[r] (bf16 bits, 80 per row) <- inputs of particle idx[r] (idx NULL: r) */
int sss_mlp_features(sss_ctx* ctx, sss_pm3* p, const sss_pm3_particles* s, const int64_t* idx, int64_t rows,
                     double rho_mean, uint16_t* X, void* stream);
/* Y[r][0..3) <- network output for input row X[r] */
int sss_mlp_forward(sss_ctx* ctx, const float* params, const uint32_t* frags, const uint16_t* X, int64_t rows,
                    float* Y, void* stream);
/* gradient of mean over rows and outputs of (Y - T)^2 with respect to the
 * parameters, over the rows idx[0..rows) of X and T (X holds x_rows rows;
 * T f32, 3 per row; idx NULL: rows 0..rows; an index outside X counts as a
 * zero row); grads (SSS_MLP_N_PARAMS f32) overwritten; loss (device f32,
 * nullable) <- the loss. Deterministic. */
int sss_mlp_grad(sss_ctx* ctx, const float* params, const uint32_t* frags, const uint16_t* X, const float* T,
                 int64_t x_rows, const int32_t* idx, int64_t rows, float* grads, float* loss, void* stream);
/* Adam (Kingma & Ba 2015) on n parameters, step t >= 1 */
int sss_mlp_adam(sss_ctx* ctx, float* params, const float* grads, float* m, float* v, int64_t n, int t,
                 double lr, double beta1, double beta2, double eps, void* stream);
/* the correction pass: a = a + out_scale * MLP(inputs) for every particle
 * of s (a holds the mesh accelerations), then the epilogue `mode` as
 * sss_pm3_gather */
int sss_mlp_correct(sss_ctx* ctx, sss_pm3* p, const sss_pm3_particles* s, const float* params,
                    const uint32_t* frags, double rho_mean, double out_scale, int mode, double hdt, double dt,
                    float* snap, void* stream);

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
 * Every call on a device shares that device's copy of the array and finds
 * the previous call's contents in it; the call clears what must start at
 * zero. Calls whose work overlaps on the same GPU (different streams with no
 * order between them) race on the array: order them on one stream. Calls on
 * different devices use separate copies of the array and do not race.
 *
 * device: CUDA device of all pointers (made current). d_status: optional
 * device int that a timed-out bounded wait sets to SSS_ERR_TIMEOUT. With
 * d_status NULL the timeout goes to an internal word that no caller can
 * read: the call still returns SSS_OK and a timed-out call's accelerations
 * may be incomplete without notice, so a caller that must detect timeouts
 * passes a d_status. errbuf/errbuf_len: optional host buffer for a message.
 * No reference counterpart. */
#define SSS_NOALLOC_SCRATCH_BYTES     (32u << 20)
#define SSS_NOALLOC_MAX_MIXED_SOURCES 1044480
int sss_allpairs_accel_noalloc(int device, int dim, int precision,
                               const double* src4, int64_t n_src,
                               const double* tgt4, int64_t n_tgt,
                               double* acc4, double eps2, int* d_status,
                               void* stream, char* errbuf, size_t errbuf_len);

/* ------------------------------------------------------------ sessions
 *
 * The state the Python classes NBodySelfGrav and NBodyCuda keep, held by the
 * library for hosts that call this ABI directly (C, C++, Go over cgo, Java
 * over JNI): host arrays in and out; the device buffers and one stream belong
 * to the session; every call is synchronous, as the reference's methods
 * return host arrays. One caller per session at a time. Errors: a status
 * code, the message (the reference's text where it has one) in
 * sss_last_error(ctx). A session lives inside its context (destroy it first). */

/* NBodySelfGrav (selfgrav_kernel.py:424-650). */
typedef struct sss_selfgrav sss_selfgrav;
/* Constructor (selfgrav_kernel.py:431-462): precision SSS_PREC_*, integrator
 * SSS_INT_*, G (the reference's G_AU = 4 pi^2 in AU^3/Msun/yr^2), Plummer
 * softening > 0 ("Softening muss positiv sein"). */
int sss_sg_create(sss_ctx* ctx, int precision, int integrator, double G, double softening,
                  sss_selfgrav** out);
void sss_sg_destroy(sss_selfgrav* s);
/* load_state (selfgrav_kernel.py:463-559): n >= 1 massive bodies, soa = host
 * f64 [2*dim][n] ([x|y|(z)|vx|vy|(vz)]), mass [n]; n_tracer massless tracers
 * in tracer_soa [2*dim][n_tracer] (NULL when none). Computes the starting
 * accelerations. */
int sss_sg_load(sss_selfgrav* s, int dim, int64_t n, const double* soa, const double* mass,
                int64_t n_tracer, const double* tracer_soa);
/* Floats per snapshot row: 2*dim*n + dim*n_tracer, the reference's row
 * [x|y|(z)|vx|vy|(vz)|tx|ty|(tz)] (selfgrav_kernel.py:600-627); 0 before a load. */
int64_t sss_sg_row_width(const sss_selfgrav* s);
/* step_batch (selfgrav_kernel.py:560-627): steps >= 1 integrator steps of
 * dt; snap_host (host f32 [steps][row]) receives the snapshot after each
 * step, or NULL for none. */
int sss_sg_step_batch(sss_selfgrav* s, double dt, int steps, float* snap_host);
/* export_f64 (selfgrav_kernel.py:629-650): out = host f64 [2*dim][n]. */
int sss_sg_export_f64(sss_selfgrav* s, double* out);

/* NBodyCuda (nbody_kernel.py:617-1060). */
typedef struct sss_nbody sss_nbody;
typedef struct sss_nbody_cfg {
    double G;             /* G_AU = 4 pi^2 */
    double softening;     /* added to r^2: SOFTENING = 1e-6 AU^2 */
    double max_sub_dt;    /* MAX_SUB_DT_YEARS = 0.5 / 365.25 */
    int    max_sub_steps; /* MAX_SUB_STEPS_PER_FRAME = 100000 */
    int    fine_guard;    /* fine-loop guard of a hot asteroid: 8000 */
    int    m_sub;         /* sub-samples per raster interval, 0..SSS_SUB_SAMPLES_MAX: 8 */
    int    pair_f32;      /* 0: f64 pair forces (the reference); 1: see sss_frame_state */
} sss_nbody_cfg;
/* Constructor (nbody_kernel.py:623-657); cfg NULL = the reference's constants. */
int sss_nbody_create(sss_ctx* ctx, const sss_nbody_cfg* cfg, sss_nbody** out);
void sss_nbody_destroy(sss_nbody* s);
/* load_state (nbody_kernel.py:659-780): n bodies, soa = host f64 [2*dim][n]
 * ([x|y|(z)|vx|vy|(vz)]), mass [n], visible and is_ast u8 [n], contact radii
 * [n] or NULL (zeros). Bodies with is_ast == 0 are the massive ones (at most
 * SSS_M_MAX: SSS_ERR_TOO_MANY_MASSIVE, "zu viele massive Koerper"). */
int sss_nbody_load(sss_nbody* s, int dim, int64_t n, const double* soa, const double* mass,
                   const unsigned char* visible, const unsigned char* is_ast, const double* radius);
/* step_batch (nbody_kernel.py:783-934): k raster samples (1..SSS_K_MAX) of
 * dt_raster in one launch; snap_host = host f32 [k][2*dim][n] in original
 * order, or NULL. SSS_ERR_GUARD when a step guard ran out (the batch is still
 * valid up to where the reference would also have stopped). */
int sss_nbody_step_batch(sss_nbody* s, double dt_raster, int k, float* snap_host);
/* st["hits"] of the last batch: the first contact of each asteroid, as
 * (asteroid index, time since the batch start, massive body index) in
 * ascending asteroid order; *n_hits = their number, at most cap written. */
int sss_nbody_hits(sss_nbody* s, int64_t* n_hits, int64_t* idx, float* t, int64_t* mas_idx, int64_t cap);
/* st["sub"][sample] of the last batch: the asteroids with a gap-free chain of
 * m_sub sub-samples (*n_hot of them, ascending) and the chains, pos = host f32
 * [m_sub][dim][n_hot]; nothing is written when n_hot > cap (ask again). */
int sss_nbody_sub(sss_nbody* s, int sample, int64_t* n_hot, int64_t* idx, float* pos, int64_t cap);
/* export_f64 (nbody_kernel.py:1042-1060): out = host f64 [2*dim][n], original order. */
int sss_nbody_export_f64(sss_nbody* s, double* out);
/* Point updates at original indices (nbody_kernel.py:947-1010): mode 0
 * apply_updates (set x, v: vals [m][2*dim]), mode 1 apply_deltas (add; idx
 * unique, "apply_deltas: idx must be unique"), mode 2 apply_body_state (set
 * x, v and mass: vals [m][2*dim+1]). Host arrays. */
int sss_nbody_scatter(sss_nbody* s, const int64_t* idx, const double* vals, int m, int mode);
/* set_radius (nbody_kernel.py:1012-1025) and deactivate_body (mass 0, not
 * visible; :1027-1040). */
int sss_nbody_set_radius(sss_nbody* s, int64_t idx, double r);
int sss_nbody_deactivate(sss_nbody* s, int64_t idx);

/* ------------------------------------------------------------ diagnostics */

/* Measured throughput of the device: kind 0 = f64 DFMA, 1 = f32 FFMA,
 * 2 = packed f32x2 FMA in TFLOP/s (2 flops per FMA lane); kind 3 = f32
 * rsqrt.approx in T operations/s (the special function unit). Synchronous;
 * the roofline denominators of the all-pairs kernels. No reference
 * counterpart. */
int sss_probe_fma(sss_ctx* ctx, int kind, int iters, double* tflops);

/* Self-test of the bounded waits: runs one wait that nothing completes, with
 * a limit of limit_s seconds (0 < limit_s <= 10), so that it gives up and
 * records SSS_ERR_TIMEOUT in the device status word, which
 * sss_device_status then returns; the context stays usable. which: 0 = the
 * mbarrier wait of the bulk-copy and tensor-core kernels (an mbarrier that
 * expects two arrivals gets one), 1 = the frame kernel's grid barrier and
 * 2 = the stream-frame kernel's grid barrier (one of two blocks leaves
 * without arriving). Asynchronous. No reference counterpart. */
int sss_selftest_wait(sss_ctx* ctx, int which, double limit_s, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SSS_H */
