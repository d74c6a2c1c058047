// Sessions of the C ABI: the state that the Python classes NBodySelfGrav
// and NBodyCuda keep (reference backend/selfgrav_kernel.py:424-650 and
// backend/nbody_kernel.py:617-1060), held by the library instead, so that a
// host without torch (C, C++, Go over cgo, Java over JNI) can drive the
// reference's call sequence load_state -> step_batch -> export_f64 / point
// updates with plain host arrays. Each session owns its device buffers and
// one stream; every call is synchronous, as the reference's methods return
// host arrays. Sessions are not thread-safe (one caller per session, as a
// Python object per session in the reference).

#include "sss_internal.cuh"

#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <new>
#include <vector>

namespace {

// Yoshida weights exactly as the Python module constants are formed
// (nbody_kernel.py:64-65: 1 / (2 - 2^(1/3)), -2^(1/3) / (2 - 2^(1/3)))
double yoshida_w1() { return 1.0 / (2.0 - pow(2.0, 1.0 / 3.0)); }
double yoshida_w0() { return -pow(2.0, 1.0 / 3.0) / (2.0 - pow(2.0, 1.0 / 3.0)); }

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

// One device allocation carved into 256-byte aligned pieces.
struct Arena {
    char* base = nullptr;
    size_t used = 0, cap = 0;
    int reserve(sss_ctx* ctx, size_t bytes) {
        release();
        if (bytes == 0) bytes = 256;
        cudaError_t e = cudaMalloc(&base, bytes);
        if (e != cudaSuccess) {
            base = nullptr;
            return sss_cuda_err(ctx, e, "cudaMalloc (session state)");
        }
        cap = bytes;
        used = 0;
        return SSS_OK;
    }
    void* take(size_t bytes) {
        void* p = base + used;
        used += al256(bytes);
        return p;
    }
    void release() {
        if (base) cudaFree(base);
        base = nullptr;
        used = cap = 0;
    }
};

__global__ void k_fill_f32(float* p, int64_t n, float v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

int sync_status(sss_ctx* ctx, cudaStream_t s) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return sss_cuda_err(ctx, e, "cudaStreamSynchronize");
    return sss_device_status(ctx, (void*)s);
}

}  // namespace

// ------------------------------------------------------------ self-gravity

struct sss_selfgrav {
    sss_ctx* ctx;
    cudaStream_t stream;
    int precision, integrator;
    double G, eps2;
    int loaded;
    sss_selfgrav_state st;
    Arena state;
    float* snap;            // device snapshots [steps][row]
    size_t snap_cap;        // floats
};

extern "C" int sss_sg_create(sss_ctx* ctx, int precision, int integrator, double G, double softening,
                             sss_selfgrav** out) {
    if (!ctx || !out) return SSS_ERR_ARG;
    *out = nullptr;
    if (!(softening > 0.0)) return sss_set_err(ctx, SSS_ERR_ARG, "Softening muss positiv sein: %g", softening);
    if (precision != SSS_PREC_F64 && precision != SSS_PREC_MIXED && precision != SSS_PREC_MIXED_TC)
        return sss_set_err(ctx, SSS_ERR_ARG, "unknown precision %d", precision);
    if (integrator != SSS_INT_KDK && integrator != SSS_INT_YOSHIDA4)
        return sss_set_err(ctx, SSS_ERR_ARG, "unknown integrator %d", integrator);
    if (!(G == G)) return sss_set_err(ctx, SSS_ERR_ARG, "G is NaN");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    sss_selfgrav* s = new (std::nothrow) sss_selfgrav();
    if (!s) return sss_set_err(ctx, SSS_ERR_CUDA, "out of host memory");
    s->ctx = ctx;
    s->precision = precision;
    s->integrator = integrator;
    s->G = G;
    s->eps2 = softening * softening;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return sss_cuda_err(ctx, e, "cudaStreamCreate (session)");
    }
    *out = s;
    return SSS_OK;
}

extern "C" void sss_sg_destroy(sss_selfgrav* s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->stream);
    s->state.release();
    if (s->snap) cudaFree(s->snap);
    cudaStreamDestroy(s->stream);
    delete s;
}

extern "C" int sss_sg_load(sss_selfgrav* s, int dim, int64_t n, const double* soa, const double* mass,
                           int64_t n_tracer, const double* tracer_soa) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (n < 1) return sss_set_err(ctx, SSS_ERR_ARG, "leerer Zustand");
    if (dim != 2 && dim != 3) return sss_set_err(ctx, SSS_ERR_ARG, "dim must be 2 or 3 (got %d)", dim);
    if (n_tracer < 0) return sss_set_err(ctx, SSS_ERR_ARG, "negative tracer count");
    if (!soa || !mass || (n_tracer > 0 && !tracer_soa)) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    const int64_t all = n + n_tracer;
    std::vector<double> hp(4 * all, 0.0), hv(4 * all, 0.0);
    for (int64_t i = 0; i < n; ++i) {
        for (int c = 0; c < dim; ++c) {
            hp[4 * i + c] = soa[c * n + i];
            hv[4 * i + c] = soa[(dim + c) * n + i];
        }
        hp[4 * i + 3] = s->G * mass[i];   // G m premultiplied (selfgrav_kernel.py:253)
    }
    for (int64_t i = 0; i < n_tracer; ++i)
        for (int c = 0; c < dim; ++c) {
            hp[4 * (n + i) + c] = tracer_soa[c * n_tracer + i];
            hv[4 * (n + i) + c] = tracer_soa[(dim + c) * n_tracer + i];
        }
    s->loaded = 0;
    const size_t rec = (size_t)all * 4 * sizeof(double);
    int rc = s->state.reserve(ctx, 4 * al256(rec));
    if (rc) return rc;
    double* p0 = (double*)s->state.take(rec);
    double* p1 = (double*)s->state.take(rec);
    double* v = (double*)s->state.take(rec);
    double* a = (double*)s->state.take(rec);
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(p0, hp.data(), rec, cudaMemcpyHostToDevice, s->stream));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(p1, hp.data(), rec, cudaMemcpyHostToDevice, s->stream));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(v, hv.data(), rec, cudaMemcpyHostToDevice, s->stream));
    SSS_CUDA_TRY(ctx, cudaMemsetAsync(a, 0, rec, s->stream));
    memset(&s->st, 0, sizeof(s->st));
    s->st.dim = dim;
    s->st.precision = s->precision;
    s->st.n_src = n;
    s->st.n_tracer = n_tracer;
    s->st.pos4[0] = p0;
    s->st.pos4[1] = p1;
    s->st.vel4 = v;
    s->st.acc4 = a;
    s->st.cur = 0;
    s->st.eps2 = s->eps2;
    rc = sss_selfgrav_init_accel(ctx, &s->st, s->stream);
    if (rc) return rc;
    rc = sync_status(ctx, s->stream);
    if (rc) return rc;
    s->loaded = 1;
    return SSS_OK;
}

extern "C" int64_t sss_sg_row_width(const sss_selfgrav* s) {
    if (!s || !s->loaded) return 0;
    return 2 * (int64_t)s->st.dim * s->st.n_src + (int64_t)s->st.dim * s->st.n_tracer;
}

extern "C" int sss_sg_step_batch(sss_selfgrav* s, double dt, int steps, float* snap_host) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!s->loaded) return sss_set_err(ctx, SSS_ERR_ARG, "kein Zustand geladen");
    if (steps < 1) return sss_set_err(ctx, SSS_ERR_ARG, "steps muss >= 1 sein: %d", steps);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    float* dsnap = nullptr;
    const size_t need = (size_t)steps * (size_t)sss_sg_row_width(s);
    if (snap_host) {
        if (need > s->snap_cap) {
            SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s->stream));
            if (s->snap) cudaFree(s->snap);
            s->snap = nullptr;
            s->snap_cap = 0;
            SSS_CUDA_TRY(ctx, cudaMalloc(&s->snap, need * sizeof(float)));
            s->snap_cap = need;
        }
        dsnap = s->snap;
    }
    int rc = sss_selfgrav_step_batch(ctx, &s->st, s->integrator, dt, steps, dsnap, s->stream);
    if (rc) return rc;
    if (snap_host)
        SSS_CUDA_TRY(ctx, cudaMemcpyAsync(snap_host, dsnap, need * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    return sync_status(ctx, s->stream);
}

extern "C" int sss_sg_export_f64(sss_selfgrav* s, double* out) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!s->loaded) return sss_set_err(ctx, SSS_ERR_ARG, "kein Zustand geladen");
    if (!out) return sss_set_err(ctx, SSS_ERR_ARG, "NULL output");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    const int64_t n = s->st.n_src;
    const int d = s->st.dim;
    std::vector<double> hp(4 * n), hv(4 * n);
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(hp.data(), s->st.pos4[s->st.cur], 4 * n * sizeof(double),
                                      cudaMemcpyDeviceToHost, s->stream));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(hv.data(), s->st.vel4, 4 * n * sizeof(double), cudaMemcpyDeviceToHost,
                                      s->stream));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s->stream));
    for (int c = 0; c < d; ++c)
        for (int64_t i = 0; i < n; ++i) {
            out[c * n + i] = hp[4 * i + c];
            out[(d + c) * n + i] = hv[4 * i + c];
        }
    return SSS_OK;
}

// -------------------------------------------- few massive + many asteroids

struct sss_nbody {
    sss_ctx* ctx;
    cudaStream_t stream;
    sss_nbody_cfg cfg;
    int loaded, dim, M, last_k;
    int64_t n, na;
    std::vector<int64_t> a_idx, m_idx;     // original indices of the asteroids / massive bodies
    std::vector<int8_t> inv_kind;          // 1 asteroid, -1 massive
    std::vector<int64_t> inv_pos;          // compact position in its group
    std::vector<double> am_h;              // asteroid masses (decide the massless mode)
    std::vector<unsigned char> avis_h;     // asteroid visibility
    sss_frame_state fs;
    Arena state;
    float* snap;                           // [K_MAX][2 dim][n]
    float* subpos;                         // [K_MAX][m_sub][dim][n_ast]
    unsigned char* subn;                   // [K_MAX][n_ast]
    float* hitt;
    int* hitm;
    int* guard;
    Arena scatter;                         // point-update staging
};

extern "C" int sss_nbody_create(sss_ctx* ctx, const sss_nbody_cfg* cfg, sss_nbody** out) {
    if (!ctx || !out) return SSS_ERR_ARG;
    *out = nullptr;
    sss_nbody_cfg c;
    if (cfg) {
        c = *cfg;
    } else {
        c.G = 4.0 * M_PI * M_PI;            // G_AU (nbody_kernel.py:60)
        c.softening = 1e-6;                 // SOFTENING
        c.max_sub_dt = 0.5 / 365.25;        // MAX_SUB_DT_YEARS
        c.max_sub_steps = 100000;           // MAX_SUB_STEPS_PER_FRAME
        c.fine_guard = SSS_FINE_GUARD;
        c.m_sub = 8;                        // SUB_SAMPLES
        c.pair_f32 = 0;
    }
    if (c.m_sub < 0 || c.m_sub > SSS_SUB_SAMPLES_MAX)
        return sss_set_err(ctx, SSS_ERR_ARG, "m_sub ausserhalb 0..%d: %d", SSS_SUB_SAMPLES_MAX, c.m_sub);
    if (c.fine_guard < 1) return sss_set_err(ctx, SSS_ERR_ARG, "fine_guard must be >= 1");
    if (c.max_sub_steps < 1) return sss_set_err(ctx, SSS_ERR_ARG, "max_sub_steps must be >= 1");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    sss_nbody* s = new (std::nothrow) sss_nbody();
    if (!s) return sss_set_err(ctx, SSS_ERR_CUDA, "out of host memory");
    s->ctx = ctx;
    s->cfg = c;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return sss_cuda_err(ctx, e, "cudaStreamCreate (session)");
    }
    *out = s;
    return SSS_OK;
}

extern "C" void sss_nbody_destroy(sss_nbody* s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->stream);
    s->state.release();
    s->scatter.release();
    cudaStreamDestroy(s->stream);
    delete s;
}

extern "C" int sss_nbody_load(sss_nbody* s, int dim, int64_t n, const double* soa, const double* mass,
                              const unsigned char* visible, const unsigned char* is_ast, const double* radius) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (dim != 2 && dim != 3) return sss_set_err(ctx, SSS_ERR_ARG, "dim must be 2 or 3 (got %d)", dim);
    if (n < 1) return sss_set_err(ctx, SSS_ERR_ARG, "leerer Zustand");
    if (!soa || !mass || !visible || !is_ast) return sss_set_err(ctx, SSS_ERR_ARG, "NULL array");
    std::vector<int64_t> a_idx, m_idx;
    for (int64_t i = 0; i < n; ++i) (is_ast[i] ? a_idx : m_idx).push_back(i);
    const int M = (int)std::min<int64_t>((int64_t)m_idx.size(), SSS_M_MAX + 1);
    if ((int64_t)m_idx.size() > SSS_M_MAX)
        return sss_set_err(ctx, SSS_ERR_TOO_MANY_MASSIVE, "zu viele massive Koerper: %lld > %d",
                           (long long)m_idx.size(), SSS_M_MAX);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    const int64_t na = (int64_t)a_idx.size();
    const int64_t na1 = na > 0 ? na : 1, m1 = M > 0 ? M : 1;
    const int ms1 = s->cfg.m_sub > 0 ? s->cfg.m_sub : 1;
    s->loaded = 0;
    size_t bytes = 0;
    bytes += 3 * 3 * al256(na1 * 8) + 3 * al256(na1 * 8) + al256(na1) + al256(na1 * 8) + al256(na1);   // ast
    bytes += 2 * 3 * al256(m1 * 8) + 2 * al256(m1 * 8) + al256(m1) + al256(m1 * 8);                    // massive
    bytes += al256((size_t)SSS_K_MAX * 2 * dim * n * 4) + al256((size_t)SSS_K_MAX * ms1 * dim * na1 * 4) +
             al256((size_t)SSS_K_MAX * na1) + al256(na1 * 4) + al256(na1 * 4) + al256(4);
    int rc = s->state.reserve(ctx, bytes);
    if (rc) return rc;
    Arena& A = s->state;
    sss_frame_state& f = s->fs;
    memset(&f, 0, sizeof(f));
    f.dim = dim;
    f.n_ast = na;
    f.M = M;
    std::vector<double> tmp(na1 > m1 ? na1 : m1);
    auto up = [&](void* dst, const void* src, size_t b) {
        return cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, s->stream);
    };
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < 3; ++c) {
        f.ast_x[c] = (double*)A.take(na1 * 8);
        f.ast_v[c] = (double*)A.take(na1 * 8);
        f.ast_acc[c] = (double*)A.take(na1 * 8);
        f.mas_x[c] = (double*)A.take(m1 * 8);
        f.mas_v[c] = (double*)A.take(m1 * 8);
        if (c < dim) {
            for (int64_t j = 0; j < na; ++j) tmp[j] = soa[c * n + a_idx[j]];
            if (na && e == cudaSuccess) e = up(f.ast_x[c], tmp.data(), na * 8);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
            for (int64_t j = 0; j < na; ++j) tmp[j] = soa[(dim + c) * n + a_idx[j]];
            if (na && e == cudaSuccess) e = up(f.ast_v[c], tmp.data(), na * 8);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
            for (int j = 0; j < M; ++j) tmp[j] = soa[c * n + m_idx[j]];
            if (M && e == cudaSuccess) e = up(f.mas_x[c], tmp.data(), (size_t)M * 8);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
            for (int j = 0; j < M; ++j) tmp[j] = soa[(dim + c) * n + m_idx[j]];
            if (M && e == cudaSuccess) e = up(f.mas_v[c], tmp.data(), (size_t)M * 8);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        }
        if (e == cudaSuccess) e = cudaMemsetAsync(f.ast_acc[c], 0, na1 * 8, s->stream);
    }
    std::vector<double> am(na1, 0.0), ar(na1, 0.0), mm(m1, 0.0), mr(m1, 0.0);
    std::vector<unsigned char> avis(na1, 0), mvis(m1, 0);
    std::vector<int64_t> aidx(na1, 0), midx(m1, 0);
    for (int64_t j = 0; j < na; ++j) {
        const int64_t i = a_idx[j];
        am[j] = mass[i];
        ar[j] = radius ? radius[i] : 0.0;
        avis[j] = visible[i] != 0;
        aidx[j] = i;
    }
    for (int j = 0; j < M; ++j) {
        const int64_t i = m_idx[j];
        mm[j] = mass[i];
        mr[j] = radius ? radius[i] : 0.0;
        mvis[j] = visible[i] != 0;
        midx[j] = i;
    }
    f.ast_m = (double*)A.take(na1 * 8);
    f.ast_vis = (unsigned char*)A.take(na1);
    f.ast_r = (double*)A.take(na1 * 8);
    f.ast_idx = (int64_t*)A.take(na1 * 8);
    f.ast_hot = (unsigned char*)A.take(na1);
    f.mas_m = (double*)A.take(m1 * 8);
    f.mas_vis = (unsigned char*)A.take(m1);
    f.mas_r = (double*)A.take(m1 * 8);
    f.mas_idx = (int64_t*)A.take(m1 * 8);
    if (e == cudaSuccess) e = up(f.ast_m, am.data(), na1 * 8);
    if (e == cudaSuccess) e = up(f.ast_vis, avis.data(), na1);
    if (e == cudaSuccess) e = up(f.ast_r, ar.data(), na1 * 8);
    if (e == cudaSuccess) e = up(f.ast_idx, aidx.data(), na1 * 8);
    if (e == cudaSuccess) e = cudaMemsetAsync(f.ast_hot, 0, na1, s->stream);
    if (e == cudaSuccess) e = up(f.mas_m, mm.data(), m1 * 8);
    if (e == cudaSuccess) e = up(f.mas_vis, mvis.data(), m1);
    if (e == cudaSuccess) e = up(f.mas_r, mr.data(), m1 * 8);
    if (e == cudaSuccess) e = up(f.mas_idx, midx.data(), m1 * 8);
    s->snap = (float*)A.take((size_t)SSS_K_MAX * 2 * dim * n * 4);
    s->subpos = (float*)A.take((size_t)SSS_K_MAX * ms1 * dim * na1 * 4);
    s->subn = (unsigned char*)A.take((size_t)SSS_K_MAX * na1);
    s->hitt = (float*)A.take(na1 * 4);
    s->hitm = (int*)A.take(na1 * 4);
    s->guard = (int*)A.take(4);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->subpos, 0, (size_t)SSS_K_MAX * ms1 * dim * na1 * 4, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->subn, 0, (size_t)SSS_K_MAX * na1, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->hitm, 0, na1 * 4, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->guard, 0, 4, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);   // the host vectors go out of scope
    if (e != cudaSuccess) return sss_cuda_err(ctx, e, "session upload");
    f.G = s->cfg.G;
    f.softening = s->cfg.softening;
    f.max_sub_dt = s->cfg.max_sub_dt;
    f.max_sub_steps = s->cfg.max_sub_steps;
    f.w1 = yoshida_w1();
    f.w0 = yoshida_w0();
    f.fine_guard = s->cfg.fine_guard;
    f.pair_f32 = s->cfg.pair_f32;
    s->dim = dim;
    s->n = n;
    s->na = na;
    s->M = M;
    s->a_idx = a_idx;
    s->m_idx = m_idx;
    s->inv_kind.assign(n, 0);
    s->inv_pos.assign(n, 0);
    for (int64_t j = 0; j < na; ++j) { s->inv_kind[a_idx[j]] = 1; s->inv_pos[a_idx[j]] = j; }
    for (int j = 0; j < M; ++j) { s->inv_kind[m_idx[j]] = -1; s->inv_pos[m_idx[j]] = j; }
    s->am_h.assign(am.begin(), am.begin() + na);
    s->avis_h.assign(avis.begin(), avis.begin() + na);
    s->last_k = 0;
    s->loaded = 1;
    return SSS_OK;
}

extern "C" int sss_nbody_step_batch(sss_nbody* s, double dt_raster, int k, float* snap_host) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!s->loaded) return sss_set_err(ctx, SSS_ERR_ARG, "kein Zustand geladen");
    if (k < 1 || k > SSS_K_MAX) return sss_set_err(ctx, SSS_ERR_ARG, "k ausserhalb 1..%d: %d", SSS_K_MAX, k);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    int massless = 1;
    for (int64_t j = 0; j < s->na; ++j)
        if (s->am_h[j] != 0.0 && s->avis_h[j] != 0) { massless = 0; break; }
    s->fs.massless_asteroids = massless;
    const int64_t na1 = s->na > 0 ? s->na : 1;
    k_fill_f32<<<(unsigned)((na1 + 255) / 256), 256, 0, s->stream>>>(s->hitt, na1, -1.0f);
    SSS_LAUNCH_CHECK(ctx, "k_fill_f32 launch");
    s->last_k = 0;
    int rc = sss_frame_launch(ctx, &s->fs, dt_raster, k, s->cfg.m_sub, s->snap, s->subpos, s->subn, s->hitt,
                              s->hitm, s->guard, s->stream);
    if (rc) return rc;
    if (snap_host)
        SSS_CUDA_TRY(ctx, cudaMemcpyAsync(snap_host, s->snap, (size_t)k * 2 * s->dim * s->n * sizeof(float),
                                          cudaMemcpyDeviceToHost, s->stream));
    rc = sync_status(ctx, s->stream);
    if (rc == SSS_OK || rc == SSS_ERR_GUARD) s->last_k = k;   // a guard stop still leaves a valid batch
    return rc;
}

extern "C" int sss_nbody_hits(sss_nbody* s, int64_t* n_hits, int64_t* idx, float* t, int64_t* mas_idx,
                              int64_t cap) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!n_hits) return sss_set_err(ctx, SSS_ERR_ARG, "NULL count");
    *n_hits = 0;
    if (!s->loaded || s->last_k == 0) return SSS_OK;
    if (s->na == 0) return SSS_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    std::vector<float> ht(s->na);
    std::vector<int> hm(s->na);
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(ht.data(), s->hitt, s->na * 4, cudaMemcpyDeviceToHost, s->stream));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(hm.data(), s->hitm, s->na * 4, cudaMemcpyDeviceToHost, s->stream));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s->stream));
    int64_t c = 0;
    for (int64_t j = 0; j < s->na; ++j) {
        if (!(ht[j] >= 0.0f)) continue;
        if (c < cap) {
            if (idx) idx[c] = s->a_idx[j];
            if (t) t[c] = ht[j];
            if (mas_idx) mas_idx[c] = (hm[j] >= 0 && hm[j] < s->M) ? s->m_idx[hm[j]] : -1;
        }
        ++c;
    }
    *n_hits = c;
    return SSS_OK;
}

extern "C" int sss_nbody_sub(sss_nbody* s, int sample, int64_t* n_hot, int64_t* idx, float* pos, int64_t cap) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!n_hot) return sss_set_err(ctx, SSS_ERR_ARG, "NULL count");
    *n_hot = 0;
    if (!s->loaded || s->last_k == 0) return sss_set_err(ctx, SSS_ERR_ARG, "no batch stepped yet");
    if (sample < 0 || sample >= s->last_k)
        return sss_set_err(ctx, SSS_ERR_ARG, "sample %d outside the last batch (k = %d)", sample, s->last_k);
    const int ms = s->cfg.m_sub, d = s->dim;
    if (ms == 0 || s->na == 0) return SSS_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    const int64_t na = s->na;
    std::vector<unsigned char> sn(na);
    std::vector<float> sp((size_t)ms * d * na);
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(sn.data(), s->subn + (size_t)sample * na, na, cudaMemcpyDeviceToHost,
                                      s->stream));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(sp.data(), s->subpos + (size_t)sample * ms * d * na, sp.size() * 4,
                                      cudaMemcpyDeviceToHost, s->stream));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s->stream));
    std::vector<int64_t> sel;
    for (int64_t j = 0; j < na; ++j)
        if (sn[j] == ms) sel.push_back(j);
    const int64_t c = (int64_t)sel.size();
    *n_hot = c;
    if (c > cap) return SSS_OK;                    // the caller asks again with room for c
    for (int64_t q = 0; q < c; ++q) {
        if (idx) idx[q] = s->a_idx[sel[q]];
        if (pos)
            for (int m = 0; m < ms; ++m)
                for (int e = 0; e < d; ++e) pos[((size_t)m * d + e) * c + q] = sp[((size_t)m * d + e) * na + sel[q]];
    }
    return SSS_OK;
}

extern "C" int sss_nbody_export_f64(sss_nbody* s, double* out) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!s->loaded) return sss_set_err(ctx, SSS_ERR_ARG, "kein Zustand geladen");
    if (!out) return sss_set_err(ctx, SSS_ERR_ARG, "NULL output");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    const int64_t n = s->n, na = s->na;
    const int d = s->dim, M = s->M;
    std::vector<double> ha(na > 0 ? na : 1), hm(M > 0 ? M : 1);
    for (int c = 0; c < 2 * d; ++c) {
        const bool vel = c >= d;
        const int e = vel ? c - d : c;
        if (na) {
            SSS_CUDA_TRY(ctx, cudaMemcpyAsync(ha.data(), vel ? s->fs.ast_v[e] : s->fs.ast_x[e], na * 8,
                                              cudaMemcpyDeviceToHost, s->stream));
        }
        if (M) {
            SSS_CUDA_TRY(ctx, cudaMemcpyAsync(hm.data(), vel ? s->fs.mas_v[e] : s->fs.mas_x[e], (size_t)M * 8,
                                              cudaMemcpyDeviceToHost, s->stream));
        }
        SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s->stream));
        for (int64_t j = 0; j < na; ++j) out[c * n + s->a_idx[j]] = ha[j];
        for (int j = 0; j < M; ++j) out[c * n + s->m_idx[j]] = hm[j];
    }
    return SSS_OK;
}

extern "C" int sss_nbody_scatter(sss_nbody* s, const int64_t* idx, const double* vals, int m, int mode) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!s->loaded) return sss_set_err(ctx, SSS_ERR_ARG, "kein Zustand geladen");
    if (mode < 0 || mode > 2) return sss_set_err(ctx, SSS_ERR_ARG, "mode must be 0, 1 or 2");
    if (m <= 0) return SSS_OK;
    if (!idx || !vals) return sss_set_err(ctx, SSS_ERR_ARG, "NULL argument");
    const int w = 2 * s->dim + (mode == 2 ? 1 : 0);
    std::vector<int64_t> slot(m);
    for (int q = 0; q < m; ++q) {
        if (idx[q] < 0 || idx[q] >= s->n)
            return sss_set_err(ctx, SSS_ERR_ARG, "index %lld outside 0..%lld", (long long)idx[q], (long long)s->n - 1);
        const int64_t p = s->inv_pos[idx[q]];
        slot[q] = s->inv_kind[idx[q]] > 0 ? p : -p - 1;
    }
    if (mode == 1) {
        std::vector<int64_t> u(idx, idx + m);
        std::sort(u.begin(), u.end());
        if (std::adjacent_find(u.begin(), u.end()) != u.end())
            return sss_set_err(ctx, SSS_ERR_ARG, "apply_deltas: idx must be unique");
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    const size_t bs = (size_t)m * 8, bv = (size_t)m * w * 8;
    if (al256(bs) + al256(bv) > s->scatter.cap) {
        int rc = s->scatter.reserve(ctx, 2 * (al256(bs) + al256(bv)));
        if (rc) return rc;
    }
    s->scatter.used = 0;
    int64_t* dslot = (int64_t*)s->scatter.take(bs);
    double* dval = (double*)s->scatter.take(bv);
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(dslot, slot.data(), bs, cudaMemcpyHostToDevice, s->stream));
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(dval, vals, bv, cudaMemcpyHostToDevice, s->stream));
    int rc = sss_frame_scatter(ctx, &s->fs, dslot, dval, m, mode, s->stream);
    if (rc) return rc;
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s->stream));
    if (mode == 2)
        for (int q = 0; q < m; ++q)
            if (s->inv_kind[idx[q]] > 0) s->am_h[s->inv_pos[idx[q]]] = vals[(size_t)q * w + w - 1];
    return SSS_OK;
}

extern "C" int sss_nbody_set_radius(sss_nbody* s, int64_t idx, double r) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!s->loaded) return sss_set_err(ctx, SSS_ERR_ARG, "kein Zustand geladen");
    if (idx < 0 || idx >= s->n) return sss_set_err(ctx, SSS_ERR_ARG, "index %lld outside the state", (long long)idx);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    const int64_t p = s->inv_pos[idx];
    double* dst = (s->inv_kind[idx] > 0 ? s->fs.ast_r : s->fs.mas_r) + p;
    SSS_CUDA_TRY(ctx, cudaMemcpyAsync(dst, &r, 8, cudaMemcpyHostToDevice, s->stream));
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s->stream));
    return SSS_OK;
}

extern "C" int sss_nbody_deactivate(sss_nbody* s, int64_t idx) {
    if (!s) return SSS_ERR_ARG;
    sss_ctx* ctx = s->ctx;
    if (!s->loaded) return sss_set_err(ctx, SSS_ERR_ARG, "kein Zustand geladen");
    if (idx < 0 || idx >= s->n) return sss_set_err(ctx, SSS_ERR_ARG, "index %lld outside the state", (long long)idx);
    if (cudaSetDevice(ctx->device) != cudaSuccess) return sss_set_err(ctx, SSS_ERR_CUDA, "cudaSetDevice failed");
    const int64_t p = s->inv_pos[idx];
    const double zero = 0.0;
    const unsigned char hidden = 0;
    if (s->inv_kind[idx] > 0) {
        SSS_CUDA_TRY(ctx, cudaMemcpyAsync(s->fs.ast_m + p, &zero, 8, cudaMemcpyHostToDevice, s->stream));
        SSS_CUDA_TRY(ctx, cudaMemcpyAsync(s->fs.ast_vis + p, &hidden, 1, cudaMemcpyHostToDevice, s->stream));
        s->am_h[p] = 0.0;
        s->avis_h[p] = 0;
    } else {
        SSS_CUDA_TRY(ctx, cudaMemcpyAsync(s->fs.mas_m + p, &zero, 8, cudaMemcpyHostToDevice, s->stream));
        SSS_CUDA_TRY(ctx, cudaMemcpyAsync(s->fs.mas_vis + p, &hidden, 1, cudaMemcpyHostToDevice, s->stream));
    }
    SSS_CUDA_TRY(ctx, cudaStreamSynchronize(s->stream));
    return SSS_OK;
}
