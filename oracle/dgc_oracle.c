/*
 * dgc_oracle.c -- FP64 CPU oracle for the cone-beam operators.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is linked by the
 * test-suite, by the smoke check and by the CPU-baseline leg of the benchmark,
 * never by the product library.  It restates, in double precision and plain C,
 * the algorithms of the reference project (TomSHINING/diff-geoCali):
 *
 *   - ray-driven forward projector:  csrc/src_cbct_forwardprojector_cuda.cu
 *       update_slab 55-83, intersect_aabb 86-112, make_source_only_ray 115-170,
 *       sample_volume_trilinear_with_grad 173-255, forward kernel 258-339;
 *     and its CPU oracle examples/check_forward_operator.py:20-105
 *       (sample count floor((exit-entry)/step)+1, t_k = entry + k*step).
 *   - analytic backward of the forward projector: same .cu file, 342-528
 *       (adjoint scatter, entry-slab chain rule 454-467, normalisation chain
 *       470-486, per-view geometry terms 488-527).
 *   - voxel-driven FDK-weighted backprojector and its backward:
 *       csrc/src_cbct_backprojector_cuda.cu 15-98 and 101-295;
 *       examples/check_operator.py:19-64 is its vectorised CPU restatement.
 *   - FDK filter: cbct_backprojector/filtering.py:54-104 (cosine preweight,
 *       zero-padded discrete Ram-Lak x Hann along U, pixel*sid/sod scale),
 *       evaluated here as the equivalent symmetric Toeplitz convolution.
 *
 * Sample-set modes of the forward projector:
 *   mode 0: the reference's FP64 CPU oracle rule (closed-form count).
 *   mode 1: the sample offsets t_k of the reference CUDA kernel, i.e. the FP32
 *           ray set-up and the FP32 recurrence t += step (fp.cu:321), after
 *           which positions, interpolation and sums are evaluated in FP64.
 *           This is "FP64 truth on the FP32 kernel's sample set".
 *
 * All arrays are C-contiguous.  Geometry is passed as 8 arrays of length A in
 * the order angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <pthread.h>
#include <unistd.h>

#define GEO_ANGLE 0
#define GEO_SID 1
#define GEO_SOD 2
#define GEO_U0 3
#define GEO_V0 4
#define GEO_SX 5
#define GEO_SY 6
#define GEO_SZ 7

/* ---- a small pthreads parallel-for (dynamic chunks of indices) ---- */
static int g_threads = 0;

int oracle_num_threads(void) {
    if (g_threads <= 0) {
        long n = sysconf(_SC_NPROCESSORS_ONLN);
        g_threads = n > 0 ? (int)n : 1;
    }
    return g_threads;
}

void oracle_set_num_threads(int n) { g_threads = n; }

typedef void (*body_fn)(long i, void* ctx);
typedef struct {
    body_fn fn;
    void* ctx;
    long n, chunk;
    long next;
} PforJob;

static void* pfor_worker(void* arg) {
    PforJob* job = (PforJob*)arg;
    for (;;) {
        long b = __atomic_fetch_add(&job->next, job->chunk, __ATOMIC_RELAXED);
        if (b >= job->n) break;
        long e = b + job->chunk < job->n ? b + job->chunk : job->n;
        for (long i = b; i < e; ++i) job->fn(i, job->ctx);
    }
    return NULL;
}

static void parallel_for(long n, long chunk, body_fn fn, void* ctx) {
    PforJob job = {fn, ctx, n, chunk > 0 ? chunk : 1, 0};
    int nt = oracle_num_threads();
    if (nt > 256) nt = 256;
    if (nt <= 1 || n <= chunk) {
        pfor_worker(&job);
        return;
    }
    pthread_t th[256];
    int started = 0;
    for (int k = 0; k < nt - 1; ++k)
        if (pthread_create(&th[started], NULL, pfor_worker, &job) == 0) ++started;
    pfor_worker(&job);
    for (int k = 0; k < started; ++k) pthread_join(th[k], NULL);
}

/* ------------------------------------------------------------------------ */
/* Forward projector                                                         */
/* ------------------------------------------------------------------------ */

typedef struct {
    double o[3];      /* ray origin (world) */
    double d[3];      /* unit direction */
    double len;       /* |T - O| */
    double tmin, tmax;
    int entry_axis;
    int hit;
    /* FP32 set-up (mode 1) */
    float of[3], df[3];
    float tminf, tmaxf;
} Ray;

/* Slab rule of fp.cu:55-112 / check_forward_operator.py:20-39, in double. */
static int slab_double(const double o[3], const double d[3], const double lo[3],
                       const double hi[3], double* tmin, double* tmax, int* axis) {
    double t0 = 0.0, t1 = INFINITY;
    int ax = -1;
    for (int k = 0; k < 3; ++k) {
        if (fabs(d[k]) < 1e-12) {
            if (!(lo[k] <= o[k] && o[k] <= hi[k])) return 0;
            continue;
        }
        double a = (lo[k] - o[k]) / d[k];
        double b = (hi[k] - o[k]) / d[k];
        if (a > b) { double tmp = a; a = b; b = tmp; }
        if (a > t0) { t0 = a; ax = k; }
        if (b < t1) t1 = b;
        if (t1 < t0) return 0;
    }
    *tmin = t0; *tmax = t1; *axis = ax;
    return 1;
}

/* The FP32 slab rule exactly as fp.cu:55-112 writes it. */
static int slab_float(const float o[3], const float d[3], const float lo[3],
                      const float hi[3], float* tmin, float* tmax, int* axis) {
    float t0 = 0.0f, t1 = FLT_MAX;
    int ax = -1;
    for (int k = 0; k < 3; ++k) {
        if (fabsf(d[k]) < 1e-12f) {
            if (!(o[k] >= lo[k] && o[k] <= hi[k])) return 0;
            continue;
        }
        volatile float inv = 1.0f / d[k];
        volatile float a = (lo[k] - o[k]) * inv;
        volatile float b = (hi[k] - o[k]) * inv;
        float aa = a, bb = b;
        if (aa > bb) { float tmp = aa; aa = bb; bb = tmp; }
        if (aa > t0) { t0 = aa; ax = k; }
        t1 = fminf(t1, bb);
        if (!(t1 >= t0)) return 0;
    }
    *tmin = t0; *tmax = t1; *axis = ax;
    return t1 >= t0;
}

static void make_ray(const double* const* g, int a, int u, int v, double px,
                     const double lo[3], const double hi[3],
                     const float lof[3], const float hif[3], int mode, Ray* r) {
    double beta = g[GEO_ANGLE][a];
    double c = cos(beta), s = sin(beta);
    double sod = g[GEO_SOD][a];
    double dn = sod - g[GEO_SID][a];
    double up = (u - g[GEO_U0][a]) * px;
    double vp = (v - g[GEO_V0][a]) * px;
    double O[3] = {-sod * s + g[GEO_SX][a], sod * c + g[GEO_SY][a], g[GEO_SZ][a]};
    double T[3] = {up * c - dn * s, up * s + dn * c, vp};
    double R[3] = {T[0] - O[0], T[1] - O[1], T[2] - O[2]};
    double len = sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
    r->hit = 0;
    r->len = len;
    for (int k = 0; k < 3; ++k) r->o[k] = O[k];
    if (mode == 0) {
        if (len <= 1e-8) return;
        for (int k = 0; k < 3; ++k) r->d[k] = R[k] / len;
        r->hit = slab_double(r->o, r->d, lo, hi, &r->tmin, &r->tmax, &r->entry_axis);
        return;
    }
    /* mode 1: FP32 set-up of fp.cu:115-170 (products fused as nvcc contracts
     * a*b+c); the geometry inputs are the float32 values given as doubles. */
    float bf = (float)beta;
    float cf = cosf(bf), sf = sinf(bf);
    float sodf = (float)sod;
    float dnf = sodf - (float)g[GEO_SID][a];
    float upf = ((float)u - (float)g[GEO_U0][a]) * (float)px;
    float vpf = ((float)v - (float)g[GEO_V0][a]) * (float)px;
    float Of[3] = {fmaf(-sodf, sf, (float)g[GEO_SX][a]), fmaf(sodf, cf, (float)g[GEO_SY][a]),
                   (float)g[GEO_SZ][a]};
    float Tf[3] = {fmaf(upf, cf, -(dnf * sf)), fmaf(upf, sf, dnf * cf), vpf};
    float Rf[3] = {Tf[0] - Of[0], Tf[1] - Of[1], Tf[2] - Of[2]};
    float lenf = sqrtf(fmaf(Rf[2], Rf[2], fmaf(Rf[1], Rf[1], Rf[0] * Rf[0])));
    if (lenf <= 1e-8f) return;
    float inv = 1.0f / lenf;
    float Df[3] = {Rf[0] * inv, Rf[1] * inv, Rf[2] * inv};
    for (int k = 0; k < 3; ++k) { r->of[k] = Of[k]; r->df[k] = Df[k]; }
    r->hit = slab_float(Of, Df, lof, hif, &r->tminf, &r->tmaxf, &r->entry_axis);
    /* FP64 evaluation uses the FP32 ray (converted exactly to double). */
    for (int k = 0; k < 3; ++k) { r->o[k] = Of[k]; r->d[k] = Df[k]; }
    r->len = lenf;
    r->tmin = r->tminf;
    r->tmax = r->tmaxf;
}

/* Number of samples and the k-th offset under the selected rule. */
static long ray_count(const Ray* r, double step, int mode) {
    if (!r->hit) return 0;
    if (mode == 0) return (long)floor((r->tmax - r->tmin) / step) + 1;
    long n = 0;
    float stepf = (float)step;
    /* bounded: a recurrence that stops advancing ends the ray */
    long cap = (long)((r->tmaxf - r->tminf) / stepf) + 4;
    for (float t = r->tminf; t <= r->tmaxf && n < cap; t += stepf) ++n;
    return n;
}

/* Trilinear sample with clamped neighbours (fp.cu:173-255), FP64. */
static inline double trilerp(const double* vol, int D, int H, int W, double x, double y,
                             double z, double grad[3], long idx[8], double w[8]) {
    double fx0 = floor(x), fy0 = floor(y), fz0 = floor(z);
    long x0r = (long)fx0, y0r = (long)fy0, z0r = (long)fz0;
    double fx = x - fx0, fy = y - fy0, fz = z - fz0;
#define CL(a, n) ((a) < 0 ? 0 : ((a) > (n) - 1 ? (n) - 1 : (a)))
    long x0 = CL(x0r, W), x1 = CL(x0r + 1, W);
    long y0 = CL(y0r, H), y1 = CL(y0r + 1, H);
    long z0 = CL(z0r, D), z1 = CL(z0r + 1, D);
#undef CL
    long plane = (long)H * W;
    long i000 = z0 * plane + y0 * W + x0, i100 = z0 * plane + y0 * W + x1;
    long i010 = z0 * plane + y1 * W + x0, i110 = z0 * plane + y1 * W + x1;
    long i001 = z1 * plane + y0 * W + x0, i101 = z1 * plane + y0 * W + x1;
    long i011 = z1 * plane + y1 * W + x0, i111 = z1 * plane + y1 * W + x1;
    double v000 = vol[i000], v100 = vol[i100], v010 = vol[i010], v110 = vol[i110];
    double v001 = vol[i001], v101 = vol[i101], v011 = vol[i011], v111 = vol[i111];
    double mx = 1 - fx, my = 1 - fy, mz = 1 - fz;
    double w000 = mx * my * mz, w100 = fx * my * mz, w010 = mx * fy * mz, w110 = fx * fy * mz;
    double w001 = mx * my * fz, w101 = fx * my * fz, w011 = mx * fy * fz, w111 = fx * fy * fz;
    if (grad) {
        grad[0] = mz * (my * (v100 - v000) + fy * (v110 - v010)) +
                  fz * (my * (v101 - v001) + fy * (v111 - v011));
        grad[1] = mz * (mx * (v010 - v000) + fx * (v110 - v100)) +
                  fz * (mx * (v011 - v001) + fx * (v111 - v101));
        grad[2] = my * (mx * (v001 - v000) + fx * (v101 - v100)) +
                  fy * (mx * (v011 - v010) + fx * (v111 - v110));
    }
    if (idx) {
        idx[0] = i000; idx[1] = i100; idx[2] = i010; idx[3] = i110;
        idx[4] = i001; idx[5] = i101; idx[6] = i011; idx[7] = i111;
        w[0] = w000; w[1] = w100; w[2] = w010; w[3] = w110;
        w[4] = w001; w[5] = w101; w[6] = w011; w[7] = w111;
    }
    return v000 * w000 + v100 * w100 + v010 * w010 + v110 * w110 + v001 * w001 +
           v101 * w101 + v011 * w011 + v111 * w111;
}

typedef struct {
    int D, H, W, A, U, V;
    double px, step, vs, off[3];
    double lo[3], hi[3];
    float lof[3], hif[3];
    int mode;
} FpCfg;

static void fp_cfg(FpCfg* c, int D, int H, int W, int A, int U, int V, double px, double step,
                   double vs, double ox, double oy, double oz, int mode) {
    c->D = D; c->H = H; c->W = W; c->A = A; c->U = U; c->V = V;
    c->px = px; c->step = step; c->vs = vs;
    c->off[0] = ox; c->off[1] = oy; c->off[2] = oz;
    int n[3] = {W, H, D};
    for (int k = 0; k < 3; ++k) {
        c->lo[k] = (-n[k] * 0.5 - 0.5) * vs + c->off[k];
        c->hi[k] = (n[k] * 0.5 - 0.5) * vs + c->off[k];
        /* fp.cu:303-312 in float (multiply-add fused) */
        c->lof[k] = fmaf(-(float)n[k] * 0.5f - 0.5f, (float)vs, (float)c->off[k]);
        c->hif[k] = fmaf((float)n[k] * 0.5f - 0.5f, (float)vs, (float)c->off[k]);
    }
    c->mode = mode;
}

static inline double sample_offset(const Ray* r, long k, double step, int mode, float* tf) {
    if (mode == 0) return r->tmin + (double)k * step;
    return (double)(*tf);
}

/* Forward projection: out[a,u,v] (fp.cu:258-339). */
typedef struct {
    FpCfg cfg;
    const double* g[8];
    const double* vol;
    const double* grad_proj;
    double* out;
    int64_t* counts;
    double* gv_views;
    double* grad_geom;
} FpJob;

static double fp_ray_value(const FpJob* j, long ray) {
    const FpCfg* c = &j->cfg;
    int V = c->V, U = c->U;
    int v = (int)(ray % V);
    int u = (int)((ray / V) % U);
    int a = (int)(ray / ((long)U * V));
    Ray r;
    make_ray(j->g, a, u, v, c->px, c->lo, c->hi, c->lof, c->hif, c->mode, &r);
    long n = ray_count(&r, c->step, c->mode);
    double acc = 0.0;
    float tf = r.tminf;
    for (long k = 0; k < n; ++k) {
        double t = sample_offset(&r, k, c->step, c->mode, &tf);
        double x = (r.o[0] + t * r.d[0] - c->off[0]) / c->vs + c->W * 0.5;
        double y = (r.o[1] + t * r.d[1] - c->off[1]) / c->vs + c->H * 0.5;
        double z = (r.o[2] + t * r.d[2] - c->off[2]) / c->vs + c->D * 0.5;
        acc += trilerp(j->vol, c->D, c->H, c->W, x, y, z, NULL, NULL, NULL);
        tf += (float)c->step;
    }
    return acc * c->step;
}

static void fp_forward_ray(long ray, void* vctx) {
    const FpJob* j = (const FpJob*)vctx;
    j->out[ray] = fp_ray_value(j, ray);
}

static void fp_job_init(FpJob* j, int D, int H, int W, const double* geom, int A, int U,
                        int V, double px, double step, double vs, double ox, double oy,
                        double oz, int mode) {
    memset(j, 0, sizeof(*j));
    fp_cfg(&j->cfg, D, H, W, A, U, V, px, step, vs, ox, oy, oz, mode);
    for (int k = 0; k < 8; ++k) j->g[k] = geom + (long)k * A;
}

void oracle_project(const double* vol, int D, int H, int W, const double* geom, int A,
                    int U, int V, double px, double step, double vs, double ox, double oy,
                    double oz, int mode, double* out) {
    FpJob j;
    fp_job_init(&j, D, H, W, geom, A, U, V, px, step, vs, ox, oy, oz, mode);
    j.vol = vol;
    j.out = out;
    parallel_for((long)A * U * V, 64, fp_forward_ray, &j);
}

/* Forward projection of a subset of rays given by flat indices (a*U+u)*V+v. */
typedef struct {
    FpJob* j;
    const int64_t* rays;
    double* out;
} FpSubJob;

static void fp_sub_ray(long i, void* vctx) {
    FpSubJob* s = (FpSubJob*)vctx;
    s->out[i] = fp_ray_value(s->j, s->rays[i]);
}

void oracle_project_rays(const double* vol, int D, int H, int W, const double* geom, int A,
                         int U, int V, double px, double step, double vs, double ox,
                         double oy, double oz, int mode, const int64_t* rays, long nrays,
                         double* out) {
    FpJob j;
    fp_job_init(&j, D, H, W, geom, A, U, V, px, step, vs, ox, oy, oz, mode);
    j.vol = vol;
    FpSubJob s = {&j, rays, out};
    parallel_for(nrays, 16, fp_sub_ray, &s);
}

static void fp_count_ray(long ray, void* vctx) {
    const FpJob* j = (const FpJob*)vctx;
    const FpCfg* c = &j->cfg;
    int V = c->V, U = c->U;
    int v = (int)(ray % V);
    int u = (int)((ray / V) % U);
    int a = (int)(ray / ((long)U * V));
    Ray r;
    make_ray(j->g, a, u, v, c->px, c->lo, c->hi, c->lof, c->hif, c->mode, &r);
    j->counts[ray] = ray_count(&r, c->step, c->mode);
}

/* Per-ray sample counts under the selected rule (for algorithmic-work figures). */
void oracle_sample_counts(int D, int H, int W, const double* geom, int A, int U, int V,
                          double px, double step, double vs, double ox, double oy, double oz,
                          int mode, int64_t* counts) {
    FpJob j;
    fp_job_init(&j, D, H, W, geom, A, U, V, px, step, vs, ox, oy, oz, mode);
    j.counts = counts;
    parallel_for((long)A * U * V, 256, fp_count_ray, &j);
}

/*
 * Per-ray trace (check_forward_operator.py:145-193 uses the same idea): a hash
 * of the entry face, the sample count and the interpolation cell of every
 * sample.  A finite difference that leaves a ray's trace unchanged stays
 * inside one smooth piece of the piecewise-smooth projector.  The hash is 0
 * ("ambiguous") when a sample coordinate lies within `margin` of a cell
 * boundary, where FP32 and FP64 evaluation may pick different cells.
 */
typedef struct {
    FpJob* j;
    double margin;
    uint64_t* out;
} TraceJob;

static inline uint64_t fnv(uint64_t h, int64_t v) {
    for (int b = 0; b < 8; ++b) {
        h ^= (uint64_t)((v >> (8 * b)) & 0xff);
        h *= 1099511628211ULL;
    }
    return h;
}

static void fp_trace_ray(long ray, void* vctx) {
    TraceJob* tj = (TraceJob*)vctx;
    const FpJob* j = tj->j;
    const FpCfg* c = &j->cfg;
    int V = c->V, U = c->U;
    int v = (int)(ray % V);
    int u = (int)((ray / V) % U);
    int a = (int)(ray / ((long)U * V));
    Ray r;
    make_ray(j->g, a, u, v, c->px, c->lo, c->hi, c->lof, c->hif, c->mode, &r);
    uint64_t h = 1469598103934665603ULL;
    long n = ray_count(&r, c->step, c->mode);
    h = fnv(h, r.hit ? r.entry_axis + 2 : 0);
    h = fnv(h, n);
    float tf = r.tminf;
    for (long k = 0; k < n; ++k) {
        double t = sample_offset(&r, k, c->step, c->mode, &tf);
        double xyz[3] = {(r.o[0] + t * r.d[0] - c->off[0]) / c->vs + c->W * 0.5,
                         (r.o[1] + t * r.d[1] - c->off[1]) / c->vs + c->H * 0.5,
                         (r.o[2] + t * r.d[2] - c->off[2]) / c->vs + c->D * 0.5};
        for (int q = 0; q < 3; ++q) {
            double f = floor(xyz[q]);
            double fr = xyz[q] - f;
            if (fr < tj->margin || fr > 1.0 - tj->margin) {
                tj->out[ray] = 0;
                return;
            }
            h = fnv(h, (int64_t)f);
        }
        tf += (float)c->step;
    }
    tj->out[ray] = h ? h : 1;
}

void oracle_ray_traces(int D, int H, int W, const double* geom, int A, int U, int V, double px,
                       double step, double vs, double ox, double oy, double oz, int mode,
                       double margin, uint64_t* out) {
    FpJob j;
    fp_job_init(&j, D, H, W, geom, A, U, V, px, step, vs, ox, oy, oz, mode);
    TraceJob tj = {&j, margin, out};
    parallel_for((long)A * U * V, 64, fp_trace_ray, &tj);
}

/*
 * Analytic backward of the forward projector (fp.cu:342-528) in FP64.
 * Work is split by view: each view owns its geometry sums (deterministic) and,
 * when the volume gradient is requested, a private buffer summed in view
 * order at the end.
 */
static void fp_backward_view(long av, void* vctx) {
    const FpJob* j = (const FpJob*)vctx;
    const FpCfg* cf = &j->cfg;
    const double* const* g = j->g;
    int a = (int)av, U = cf->U, V = cf->V, D = cf->D, H = cf->H, W = cf->W;
    double px = cf->px, step = cf->step, vs = cf->vs;
    long nvox = (long)D * H * W;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double* gv = j->gv_views ? j->gv_views + (long)a * nvox : NULL;
    double beta = g[GEO_ANGLE][a];
    double c = cos(beta), s = sin(beta);
    double sod = g[GEO_SOD][a];
    double dn = sod - g[GEO_SID][a];
    if (cf->mode == 1) {
        /* the FP32 kernel's per-view terms (fp.cu:488-493) */
        float bf = (float)beta;
        c = cosf(bf);
        s = sinf(bf);
        dn = (double)((float)sod - (float)g[GEO_SID][a]);
    }
    for (int u = 0; u < U; ++u) {
        for (int v = 0; v < V; ++v) {
            double go = j->grad_proj[((long)a * U + u) * V + v];
            if (go == 0.0) continue; /* fp.cu:381 */
            Ray r;
            make_ray(g, a, u, v, px, cf->lo, cf->hi, cf->lof, cf->hif, cf->mode, &r);
            if (!(r.len > 1e-8)) continue;
            double god[3] = {0, 0, 0}, gdir[3] = {0, 0, 0};
            if (r.hit) {
                long n = ray_count(&r, step, cf->mode);
                double gs = go * step;
                double gtmin = 0.0;
                float tf = r.tminf;
                for (long k = 0; k < n; ++k) {
                    double t = sample_offset(&r, k, step, cf->mode, &tf);
                    double x = (r.o[0] + t * r.d[0] - cf->off[0]) / vs + W * 0.5;
                    double y = (r.o[1] + t * r.d[1] - cf->off[1]) / vs + H * 0.5;
                    double z = (r.o[2] + t * r.d[2] - cf->off[2]) / vs + D * 0.5;
                    double gr[3];
                    long idx[8];
                    double w[8];
                    trilerp(j->vol, D, H, W, x, y, z, gr, idx, w);
                    if (gv)
                        for (int q = 0; q < 8; ++q) gv[idx[q]] += gs * w[q];
                    double gw[3] = {gr[0] / vs, gr[1] / vs, gr[2] / vs};
                    for (int q = 0; q < 3; ++q) {
                        god[q] += gs * gw[q];
                        gdir[q] += gs * gw[q] * t;
                    }
                    gtmin += gs * (gw[0] * r.d[0] + gw[1] * r.d[1] + gw[2] * r.d[2]);
                    tf += (float)step;
                }
                int e = r.entry_axis;
                if (e >= 0) {
                    god[e] -= gtmin / r.d[e];
                    gdir[e] -= gtmin * r.tmin / r.d[e];
                }
            }
            double ddg = r.d[0] * gdir[0] + r.d[1] * gdir[1] + r.d[2] * gdir[2];
            double gray[3], gorig[3];
            for (int q = 0; q < 3; ++q) {
                gray[q] = (gdir[q] - r.d[q] * ddg) / r.len;
                gorig[q] = god[q] - gray[q];
            }
            double up = (u - g[GEO_U0][a]) * px;
            double dOx = -sod * c, dOy = -sod * s;
            double dTx = -up * s - dn * c, dTy = up * c - dn * s;
            acc[GEO_ANGLE] += gorig[0] * dOx + gorig[1] * dOy + gray[0] * dTx + gray[1] * dTy;
            acc[GEO_SID] += gray[0] * s - gray[1] * c;
            acc[GEO_SOD] += (gorig[0] + gray[0]) * (-s) + (gorig[1] + gray[1]) * c;
            acc[GEO_U0] += -px * (gray[0] * c + gray[1] * s);
            acc[GEO_V0] += -px * gray[2];
            acc[GEO_SX] += gorig[0];
            acc[GEO_SY] += gorig[1];
            acc[GEO_SZ] += gorig[2];
        }
    }
    for (int k = 0; k < 8; ++k) j->grad_geom[(long)k * cf->A + a] = acc[k];
}

typedef struct {
    double* dst;
    const double* views;
    long nvox;
    int A;
} SumViewsJob;

static void sum_views_voxel(long i, void* vctx) {
    const SumViewsJob* j = (const SumViewsJob*)vctx;
    double acc = 0.0;
    for (int a = 0; a < j->A; ++a) acc += j->views[(long)a * j->nvox + i];
    j->dst[i] = acc;
}

/* grad_vol (may be NULL) has shape [D,H,W]; grad_geom is [8][A]. */
void oracle_project_backward(const double* grad_proj, const double* vol, int D, int H,
                             int W, const double* geom, int A, int U, int V, double px,
                             double step, double vs, double ox, double oy, double oz,
                             int mode, double* grad_vol, double* grad_geom) {
    FpJob j;
    fp_job_init(&j, D, H, W, geom, A, U, V, px, step, vs, ox, oy, oz, mode);
    long nvox = (long)D * H * W;
    j.vol = vol;
    j.grad_proj = grad_proj;
    j.grad_geom = grad_geom;
    if (grad_vol) j.gv_views = (double*)calloc((size_t)A * nvox, sizeof(double));
    parallel_for(A, 1, fp_backward_view, &j);
    if (grad_vol) {
        SumViewsJob sj = {grad_vol, j.gv_views, nvox, A};
        parallel_for(nvox, 4096, sum_views_voxel, &sj);
        free(j.gv_views);
    }
}

/* ------------------------------------------------------------------------ */
/* Backprojector                                                             */
/* ------------------------------------------------------------------------ */

typedef struct {
    int valid;
    double u_idx, v_idx, w, t, q, l, m, px, py, ds_u, ds_n, du, dv;
} BpTerm;

/* Per voxel-view mapping of bp.cu:43-75 (and check_operator.py:34-51). */
static inline void bp_term(const double* const* g, int a, double vx, double vy, double vz,
                           double pix, int U, int V, BpTerm* b) {
    double beta = g[GEO_ANGLE][a];
    double c = cos(beta), s = sin(beta);
    double px = vx * c + vy * s, py = -vx * s + vy * c, pz = vz;
    double sx = g[GEO_SX][a], sy = g[GEO_SY][a];
    double ds_u = sx * c + sy * s, ds_n = -sx * s + sy * c, ds_v = g[GEO_SZ][a];
    double sod = g[GEO_SOD][a], sid = g[GEO_SID][a];
    double q = sod + ds_n - py, l = sid + ds_n;
    b->valid = 0;
    if (q <= 1e-6 || l <= 1e-6) return;
    double t = l / q;
    double up = ds_u + t * (px - ds_u), vp = ds_v + t * (pz - ds_v);
    double m = sod + ds_n;
    double ui = up / pix + g[GEO_U0][a], vi = vp / pix + g[GEO_V0][a];
    if (!(ui >= 0.0 && ui < U - 1.0 && vi >= 0.0 && vi < V - 1.0)) return;
    b->valid = 1;
    b->u_idx = ui; b->v_idx = vi; b->w = (m / q) * (m / q); b->t = t;
    b->q = q; b->l = l; b->m = m; b->px = px; b->py = py; b->ds_u = ds_u; b->ds_n = ds_n;
    b->du = px - ds_u; b->dv = pz - ds_v;
}

typedef struct {
    const double* g[8];
    const double* proj;
    const double* grad_vol;
    double* vol;
    double* grad_proj;
    double* grad_geom;
    int A, U, V, D, H, W;
    double pix, vs, off[3];
} BpJob;

static void bp_forward_row(long zy, void* vctx) {
    const BpJob* j = (const BpJob*)vctx;
    int z = (int)(zy / j->H), y = (int)(zy % j->H);
    double vz = (z - j->D * 0.5) * j->vs + j->off[2];
    double vy = (y - j->H * 0.5) * j->vs + j->off[1];
    for (int x = 0; x < j->W; ++x) {
        double vx = (x - j->W * 0.5) * j->vs + j->off[0];
        double acc = 0.0;
        for (int a = 0; a < j->A; ++a) {
            BpTerm b;
            bp_term(j->g, a, vx, vy, vz, j->pix, j->U, j->V, &b);
            if (!b.valid) continue;
            long u0 = (long)floor(b.u_idx), v0 = (long)floor(b.v_idx);
            double fu = b.u_idx - u0, fv = b.v_idx - v0;
            const double* img = j->proj + (long)a * j->U * j->V;
            long V = j->V;
            double p00 = img[u0 * V + v0], p10 = img[(u0 + 1) * V + v0];
            double p01 = img[u0 * V + v0 + 1], p11 = img[(u0 + 1) * V + v0 + 1];
            acc += b.w * ((1 - fu) * (1 - fv) * p00 + fu * (1 - fv) * p10 +
                          (1 - fu) * fv * p01 + fu * fv * p11);
        }
        j->vol[((long)z * j->H + y) * j->W + x] = acc;
    }
}

static void bp_job_init(BpJob* j, int A, int U, int V, const double* geom, double pix, int D,
                        int H, int W, double vs, double ox, double oy, double oz) {
    memset(j, 0, sizeof(*j));
    for (int k = 0; k < 8; ++k) j->g[k] = geom + (long)k * A;
    j->A = A; j->U = U; j->V = V; j->D = D; j->H = H; j->W = W;
    j->pix = pix; j->vs = vs; j->off[0] = ox; j->off[1] = oy; j->off[2] = oz;
}

/* vol[z,y,x] = sum_a mask * w * bilerp (bp.cu:15-98). */
void oracle_backproject(const double* proj, int A, int U, int V, const double* geom,
                        double pix, int D, int H, int W, double vs, double ox, double oy,
                        double oz, double* vol) {
    BpJob j;
    bp_job_init(&j, A, U, V, geom, pix, D, H, W, vs, ox, oy, oz);
    j.proj = proj;
    j.vol = vol;
    parallel_for((long)D * H, 1, bp_forward_row, &j);
}

/* Backward of the backprojector (bp.cu:101-295) in FP64, split by view. */
static void bp_backward_view(long av, void* vctx) {
    const BpJob* j = (const BpJob*)vctx;
    int a = (int)av, U = j->U, D = j->D, H = j->H, W = j->W;
    long V = j->V;
    double pix = j->pix, vs = j->vs;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const double* img = j->proj + (long)a * U * V;
    double* gimg = j->grad_proj + (long)a * U * V;
    double beta = j->g[GEO_ANGLE][a];
    double c = cos(beta), s = sin(beta);
    for (int z = 0; z < D; ++z)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                double gval = j->grad_vol[((long)z * H + y) * W + x];
                double vx = (x - W * 0.5) * vs + j->off[0], vy = (y - H * 0.5) * vs + j->off[1];
                double vz = (z - D * 0.5) * vs + j->off[2];
                BpTerm b;
                bp_term(j->g, a, vx, vy, vz, pix, U, (int)V, &b);
                if (!b.valid) continue;
                long u0 = (long)floor(b.u_idx), v0 = (long)floor(b.v_idx);
                double fu = b.u_idx - u0, fv = b.v_idx - v0;
                double p00 = img[u0 * V + v0], p10 = img[(u0 + 1) * V + v0];
                double p01 = img[u0 * V + v0 + 1], p11 = img[(u0 + 1) * V + v0 + 1];
                double interp = (1 - fu) * (1 - fv) * p00 + fu * (1 - fv) * p10 +
                                (1 - fu) * fv * p01 + fu * fv * p11;
                double Iu = (1 - fv) * (p10 - p00) + fv * (p11 - p01);
                double Iv = (1 - fu) * (p01 - p00) + fu * (p11 - p10);
                double gb = gval * b.w;
                gimg[u0 * V + v0] += gb * (1 - fu) * (1 - fv);
                gimg[(u0 + 1) * V + v0] += gb * fu * (1 - fv);
                gimg[u0 * V + v0 + 1] += gb * (1 - fu) * fv;
                gimg[(u0 + 1) * V + v0 + 1] += gb * fu * fv;
                double iq = 1.0 / b.q, iq2 = iq * iq, iq3 = iq2 * iq, m2 = b.m * b.m;
                double ip = 1.0 / pix;
                /* sid moves only the detector plane (bp.cu:213-219) */
                acc[GEO_SID] += gval * b.w * (Iu * b.du * iq + Iv * b.dv * iq) * ip;
                /* sod moves source and detector radially (bp.cu:221-230) */
                double dt = -b.l * iq2;
                double dW = 2 * b.m * iq2 - 2 * m2 * iq3;
                acc[GEO_SOD] += gval * (dW * interp + b.w * (Iu * b.du * dt + Iv * b.dv * dt) * ip);
                /* beta rotates the point and the source offset (bp.cu:232-250) */
                double dpx = b.py, dsu = b.ds_n, dsn = -b.ds_u;
                double dq = b.px - b.ds_u;
                double dtb = (dsn * b.q - b.l * dq) * iq2;
                double dU = (1 - b.t) * dsu + b.t * dpx + b.du * dtb;
                double dV = b.dv * dtb;
                double dWb = 2 * b.m * iq2 * dsn - 2 * m2 * iq3 * dq;
                acc[GEO_ANGLE] += gval * (dWb * interp + b.w * (Iu * dU + Iv * dV) * ip);
                acc[GEO_U0] += gval * b.w * Iu;
                acc[GEO_V0] += gval * b.w * Iv;
                /* world source offsets (bp.cu:255-292) */
                double dsus[2] = {c, s}, dsns[2] = {-s, c};
                for (int k = 0; k < 2; ++k) {
                    double dtk = dsns[k] * (b.q - b.l) * iq2;
                    double dUk = (1 - b.t) * dsus[k] + b.du * dtk;
                    double dVk = b.dv * dtk;
                    double dWk = 2 * b.m * iq2 * dsns[k] - 2 * m2 * iq3 * dsns[k];
                    acc[GEO_SX + k] += gval * (dWk * interp + b.w * (Iu * dUk + Iv * dVk) * ip);
                }
                acc[GEO_SZ] += gval * b.w * Iv * (1 - b.t) * ip;
            }
    for (int k = 0; k < 8; ++k) j->grad_geom[(long)k * j->A + a] = acc[k];
}

void oracle_backproject_backward(const double* grad_vol, const double* proj, int A, int U,
                                 int V, const double* geom, double pix, int D, int H, int W,
                                 double vs, double ox, double oy, double oz,
                                 double* grad_proj, double* grad_geom) {
    BpJob j;
    bp_job_init(&j, A, U, V, geom, pix, D, H, W, vs, ox, oy, oz);
    j.proj = proj;
    j.grad_vol = grad_vol;
    j.grad_proj = grad_proj;
    j.grad_geom = grad_geom;
    memset(grad_proj, 0, sizeof(double) * (size_t)A * U * V);
    parallel_for(A, 1, bp_backward_view, &j);
}

/* ------------------------------------------------------------------------ */
/* FDK filter                                                                */
/* ------------------------------------------------------------------------ */

/*
 * Taps h[0..U-1] of the filter of filtering.py:87-103 as a symmetric
 * Toeplitz kernel: with P = 2^bitlen(2U-1), H[k] = Re(DFT_P(r))[k] * hann[k],
 * h = IDFT_P(H) (real and even).  r is the discrete Ram-Lak kernel
 * r[0] = 1/(4 px^2), r[n odd] = -1/(pi n px)^2 (n taken in (-P/2, P/2]);
 * hann[k] = 0.5+0.5cos(2 pi f/alpha) for |f| <= alpha/2 (f = fftfreq), else 0.
 * Direct O(P^2) sums in FP64.
 */
void oracle_fdk_taps(int U, double px, double alpha, double* h) {
    int P = 1;
    {
        int n = 2 * U - 1, bl = 0;
        while (n) { ++bl; n >>= 1; }
        P = 1 << bl;
    }
    double* cs = (double*)malloc(sizeof(double) * P);
    for (int j = 0; j < P; ++j) cs[j] = cos(2.0 * M_PI * (double)j / (double)P);
    double* H = (double*)malloc(sizeof(double) * P);
    for (int k = 0; k < P; ++k) {
        double R = 1.0 / (4.0 * px * px);
        for (int n = 1; n < P; ++n) {
            int nn = n > P / 2 ? n - P : n;
            if (nn % 2 == 0) continue;
            double rn = -1.0 / ((M_PI * nn * px) * (M_PI * nn * px));
            R += rn * cs[(long)k * n % P];
        }
        double f = (k <= (P - 1) / 2 ? k : k - P) / (double)P;
        double hann = fabs(f) <= alpha * 0.5 ? 0.5 + 0.5 * cos(2.0 * M_PI * f / alpha) : 0.0;
        H[k] = R * hann;
    }
    for (int m = 0; m < U; ++m) {
        double acc = 0.0;
        for (int k = 0; k < P; ++k) acc += H[k] * cs[(long)k * m % P];
        h[m] = acc / P;
    }
    free(cs);
    free(H);
}

typedef struct {
    const double* proj;
    const double* sod;
    const double* sid;
    const double* h;
    double* out;
    int A, U, V;
    double px;
    const double* frame_dist; /* [A] or NULL: sid */
    const double* frame_u;    /* [A] or NULL: (U-1)/2 */
    const double* frame_v;    /* [A] or NULL: (V-1)/2 */
} FdkJob;

static void fdk_column(long av, void* vctx) {
    const FdkJob* j = (const FdkJob*)vctx;
    int a = (int)(av / j->V), v = (int)(av % j->V), U = j->U;
    long V = j->V;
    double* wcol = (double*)malloc(sizeof(double) * U);
    double sid = j->sid[a], sod = j->sod[a];
    double dn = j->frame_dist ? j->frame_dist[a] : sid;
    double cu = j->frame_u ? j->frame_u[a] : (U - 1) / 2.0;
    double cv = j->frame_v ? j->frame_v[a] : (V - 1) / 2.0;
    double vv = (v - cv) * j->px;
    for (int k = 0; k < U; ++k) {
        double uu = (k - cu) * j->px;
        double dist = sqrt(dn * dn + uu * uu + vv * vv);
        wcol[k] = j->proj[((long)a * U + k) * V + v] * (dn / dist);
    }
    for (int u = 0; u < U; ++u) {
        double acc = 0.0;
        for (int k = 0; k < U; ++k) acc += j->h[u > k ? u - k : k - u] * wcol[k];
        j->out[((long)a * U + u) * V + v] = acc * j->px * (sid / sod);
    }
    free(wcol);
}

/*
 * fdk_filter (filtering.py:54-104): out = [sum_k h[|u-k|] * p[k,v] * sid/dist(k,v)]
 * * px * sid/sod, per view; sid/sod are per-view arrays [A].  The preweight
 * frame (frame_dist, frame_u, frame_v; each NULL for the centred default of
 * filtering.py:82-85) replaces sid and the array centre inside the cosine
 * weight: dn / sqrt(dn^2 + ((k-fu) px)^2 + ((v-fv) px)^2), no counterpart in
 * the reference.
 */
void oracle_fdk_filter_frame(const double* proj, int A, int U, int V, double px,
                             const double* sod, const double* sid, const double* frame_dist,
                             const double* frame_u, const double* frame_v, double alpha,
                             double* out) {
    double* h = (double*)malloc(sizeof(double) * U);
    oracle_fdk_taps(U, px, alpha, h);
    FdkJob j = {proj, sod, sid, h, out, A, U, V, px, frame_dist, frame_u, frame_v};
    parallel_for((long)A * V, 4, fdk_column, &j);
    free(h);
}

void oracle_fdk_filter(const double* proj, int A, int U, int V, double px, const double* sod,
                       const double* sid, double alpha, double* out) {
    oracle_fdk_filter_frame(proj, A, U, V, px, sod, sid, NULL, NULL, NULL, alpha, out);
}
