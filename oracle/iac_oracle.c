/*
 * iac_oracle.c -- CPU restatement of IncohAutoCorrelate's pair-correlation path.
 *
 * TEST INFRASTRUCTURE ONLY (see iac_oracle.h).  Nothing in the product links
 * this file; it is the checker the CUDA kernels are compared against.
 *
 * Build: gcc -O2 -std=c11 -ffp-contract=off -fopenmp -fPIC -shared (oracle/Makefile).
 * -ffp-contract=off keeps every a*b+c as a rounded multiply followed by a
 * rounded add, which is the operation order the reference's source spells out.
 *
 * Citations are path:line inside the FabianTr/IncohAutoCorrelate tree,
 * IAC/ = IncohAutoCorrelate/.
 */
#include "iac_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static inline void add_u64(uint64_t *p, uint64_t v) { __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }

/* Settings::FloatToInt(float), IAC/Settings.h:168-171 */
static inline long float_to_int_f(float f, float step, float offset)
{
    return (long)floorf(((f + offset) / step) + 0.5f);
}
/* Settings::FloatToInt(double), IAC/Settings.h:172-175 */
static inline long float_to_int_d(double f, float step, float offset)
{
    return (long)floor(((f + (double)offset) / (double)step) + 0.5);
}

/* ===================================================================== */
/* geometry                                                              */
/* ===================================================================== */

/* Detector::Calc_kMap, IAC/Detector.cpp:310-361: unit vectors r/|r| and the
 * per-axis extent Max_q = |max k - min k|. */
void iaco_calc_kmap(const float *pm, uint64_t npix, float *kmap, float max_q[3])
{
    float mx[3] = {-100.0f, -100.0f, -100.0f};
    float mn[3] = {100.0f, 100.0f, 100.0f};
    for (uint64_t i = 0; i < npix; i++) {
        float x = pm[3 * i + 0], y = pm[3 * i + 1], z = pm[3 * i + 2];
        float r = sqrtf(x * x + y * y + z * z);
        x = x / r;
        y = y / r;
        z = z / r;
        kmap[3 * i + 0] = x;
        kmap[3 * i + 1] = y;
        kmap[3 * i + 2] = z;
        if (x > mx[0]) mx[0] = x;
        if (y > mx[1]) mx[1] = y;
        if (z > mx[2]) mx[2] = z;
        if (x < mn[0]) mn[0] = x;
        if (y < mn[1]) mn[1] = y;
        if (z < mn[2]) mn[2] = z;
    }
    for (int d = 0; d < 3; d++) max_q[d] = fabsf(mx[d] - mn[d]);
}

/* Simulator::GeneratePixelMap, IAC/Simulator.cpp:495-519.  Layout
 * PixelMap[3*a*SizeB + 3*b + d]; a is the slow axis. */
void iaco_generate_pixel_map(int size_a, int size_b, float pixel_size, const float center[3],
                             const float vec_a_in[3], const float vec_b_in[3], float *pm)
{
    float va[3] = {vec_a_in[0], vec_a_in[1], vec_a_in[2]};
    float vb[3] = {vec_b_in[0], vec_b_in[1], vec_b_in[2]};
    float na = sqrtf(va[0] * va[0] + va[1] * va[1] + va[2] * va[2]);
    for (int d = 0; d < 3; d++) va[d] = va[d] / na;
    float nb = sqrtf(vb[0] * vb[0] + vb[1] * vb[1] + vb[2] * vb[2]);
    for (int d = 0; d < 3; d++) vb[d] = vb[d] / nb;
    for (int a = 0; a < size_a; a++)
        for (int b = 0; b < size_b; b++)
            for (int d = 0; d < 3; d++)
                pm[3 * (size_t)a * size_b + 3 * (size_t)b + d] =
                    (float)(center[d] + va[d] * pixel_size * (a - 0.5 * size_a) +
                            vb[d] * pixel_size * (b - 0.5 * size_b));
}

/* voxel pitch shared by all mesh constructors, e.g. IAC/ACMesh.cpp:96-101 */
static void mesh_pitch(iaco_mesh_shape *s, float maxq)
{
    s->max_q = maxq;
    s->dq_per_voxel = maxq / (float)(((s->size_ab - 1) / 2) - 2);
    s->voxel_per_dq = (uint32_t)floorf(1.0f / s->dq_per_voxel);
    s->dq_per_voxel = 1.0f / ((float)s->voxel_per_dq);
}

/* ACMesh::CreateBigMeshForDetector, IAC/ACMesh.cpp:74-106 (identical sizing in
 * CreateBigMesh_CofQ_ForDetector, :107-139).  Returns -1 for an even edge,
 * which the reference rejects with std::invalid_argument. */
int iaco_big_mesh_shape(const float mq[3], int edge, float q_zoom, iaco_mesh_shape *s)
{
    if (edge % 2 == 0) return -1;
    s->k_a = 0;
    s->k_b = 1;
    s->k_c = 2;
    s->size_ab = (uint32_t)edge + 2;
    s->size_c = s->size_ab;
    s->center[0] = s->center[1] = (s->size_ab - 1) / 2;
    s->center[2] = (s->size_c - 1) / 2;
    float m = mq[0] > mq[1] ? mq[0] : mq[1];
    m = m > mq[2] ? m : mq[2];
    mesh_pitch(s, m / q_zoom);
    return 0;
}

/* ACMesh::CreateSmallMesh_CofQ_ForDetector, IAC/ACMesh.cpp:140-206 */
int iaco_small_cq_mesh_shape(const float mq[3], int perp, float q_zoom, iaco_mesh_shape *s)
{
    if (perp % 2 == 0) return -1;
    uint32_t a = 0, b = 1, c = 2, t;
    if (mq[b] > mq[a]) { t = a; a = b; b = t; }
    if (mq[c] > mq[b]) { t = c; c = b; b = t; }
    if (mq[b] > mq[a]) { t = a; a = b; b = t; }
    s->k_a = a;
    s->k_b = b;
    s->k_c = c;
    s->size_ab = (uint32_t)perp + 2;
    if (q_zoom == 1.0f)
        s->size_c = (uint32_t)(int)floor((double)((mq[c] / mq[a]) * (float)perp) + 2.5);
    else
        s->size_c = s->size_ab;
    if (s->size_c % 2 == 0) s->size_c += 1;
    s->center[0] = s->center[1] = (s->size_ab - 1) / 2;
    s->center[2] = (s->size_c - 1) / 2;
    mesh_pitch(s, mq[a] / q_zoom);
    return 0;
}

/* AC1D::Initialize(Det, ArraySize, QZoom), IAC/AC1D.cpp:53-59 */
void iaco_ac1d_shape_init(const float mq[3], uint32_t size, float q_zoom, iaco_ac1d_shape *s)
{
    s->size = size;
    s->max_q = sqrtf(mq[0] * mq[0] + mq[1] * mq[1] + mq[2] * mq[2]) / q_zoom;
    s->dq_per_step = s->max_q / ((float)(size - 2));
}

/* ===================================================================== */
/* photonisation                                                         */
/* ===================================================================== */

/* ArrayOperators::DiscretizeToPhotons, IAC/ArrayOperators.h:138-148 */
void iaco_discretize_to_photons(float *a, uint64_t n, float thr, float step)
{
    for (uint64_t i = 0; i < n; i++) a[i] = ceilf((a[i] - thr) / step) * (float)(a[i] >= thr);
}

/* Detector::LoadAndAverageIntensity, IAC/Detector.cpp:687-790, for a batch of
 * loaded frames (events in order): mask (ParMultiplyElementwise,
 * IAC/ArrayOperators.h:118-125); without discretisation zero values below a
 * positive threshold and add values >= threshold to the running intensity
 * (ParAdd with threshold, IAC/ArrayOperators.h:75-86); with a sampling step
 * discretise (DiscretizeToPhotones, IAC/Detector.cpp:90-96) and add
 * (long)floor(v + 0.5) to the per-pixel count; per event the sequential FP32
 * Sum (IAC/ArrayOperators.h:259-267) gives MeanIntensity = Sum / npix and the
 * photon sum.  sum / discr accumulate across calls. */
void iaco_average_frames(const float *frames, uint64_t npix, uint32_t nframes, const int32_t *mask,
                         float thr, float step, float *sum, int64_t *discr, float *mean_intensity,
                         float *photon_sum)
{
    float *tmp = (float *)malloc(sizeof(float) * npix);
    for (uint32_t f = 0; f < nframes; f++) {
        const float *fr = frames + (size_t)f * npix;
        for (uint64_t j = 0; j < npix; j++) tmp[j] = mask ? fr[j] * (float)mask[j] : fr[j];
        if (step <= 0) {
            if (thr > 0)
                for (uint64_t j = 0; j < npix; j++)
                    if (tmp[j] < thr) tmp[j] = 0.0f;
            for (uint64_t j = 0; j < npix; j++)
                if (tmp[j] >= thr) sum[j] += tmp[j];
        } else {
            for (uint64_t j = 0; j < npix; j++) {
                if (tmp[j] >= thr) {
                    iaco_discretize_to_photons(&tmp[j], 1, thr, step);
                    discr[j] += (int64_t)floor(tmp[j] + 0.5);
                } else {
                    tmp[j] = 0;
                }
            }
        }
        float s = 0.0f;
        for (uint64_t j = 0; j < npix; j++) s += tmp[j];
        mean_intensity[f] = s / ((float)npix);
        if (photon_sum && step > 0) photon_sum[f] = s;
    }
    free(tmp);
}

/* the end of LoadAndAverageIntensity: Intensity = (float)count (discretised)
 * or the running sum, times 1 / nframes (ParMultiplyScalar) */
void iaco_average_finish(const float *sum, const int64_t *discr, uint64_t npix, uint32_t nframes_total,
                         float *intensity)
{
    const float f = 1.0f / ((float)nframes_total);
    for (uint64_t j = 0; j < npix; j++) intensity[j] = (discr ? (float)discr[j] : sum[j]) * f;
}

/* Detector::CreateSparseHitList(Threshold[, Step]), IAC/Detector.cpp:926-958:
 * keep pixels with I >= Threshold and I > 0 in pixel order, then photonise the
 * value.  out4 receives (kx, ky, kz, value) per kept pixel. */
uint64_t iaco_sparse_hitlist(const float *I, const float *kmap, uint64_t npix, float thr,
                             float step, int photonize, float *out4)
{
    uint64_t n = 0;
    for (uint64_t i = 0; i < npix; i++) {
        float v = I[i];
        if (v >= thr && v > 0) {
            out4[4 * n + 0] = kmap[3 * i + 0];
            out4[4 * n + 1] = kmap[3 * i + 1];
            out4[4 * n + 2] = kmap[3 * i + 2];
            if (photonize) iaco_discretize_to_photons(&v, 1, thr, step);
            out4[4 * n + 3] = v;
            n++;
        }
    }
    return n;
}

/* ===================================================================== */
/* (a) sparse photon pairs                                               */
/* ===================================================================== */

typedef struct {
    uint64_t *ac;
    int S, C, half_ss;
    double mult;
    uint64_t oob;
} halfmesh_t;

/* AddQToPositiveSS, IAC/kernel.cl:349-372.  The reference performs no range
 * check; here an index outside the half mesh is counted and skipped (it can
 * only occur for rotation matrices that are not orthonormal). */
static void hm_put(halfmesh_t *h, int fs, int ms, int ss, uint64_t v)
{
    if (fs < 0 || ms < 0 || ss < 0 || fs >= h->S || ms >= h->S || ss >= h->half_ss) {
        __atomic_fetch_add(&h->oob, 1, __ATOMIC_RELAXED);
        return;
    }
    add_u64(&h->ac[(size_t)fs + (size_t)ms * h->S + (size_t)ss * h->S * h->S], v);
}
static void add_q_to_positive_ss(halfmesh_t *h, int fs, int ms, int ss, uint64_t val, int qzero)
{
    if (ss > 0) {
        hm_put(h, fs, ms, ss, val);
    } else {
        if (ss == 0) hm_put(h, fs, ms, ss, val);
        if (!qzero) hm_put(h, 2 * h->C - fs, 2 * h->C - ms, 0 - ss, val);
    }
}

/* AddRotatedQToMesh, IAC/kernel.cl:374-448 */
static void add_rotated_q(halfmesh_t *h, double val, float q0, float q1, float q2, int interp2,
                          int qzero)
{
    const int C = h->C;
    if (interp2 == 0) {
        uint64_t v = (uint64_t)(val * h->mult);
        int fs = (int)((float)C + roundf(q0));
        int ms = (int)((float)C + roundf(q1));
        int ss = (int)(roundf(q2));
        add_q_to_positive_ss(h, fs, ms, ss, v, qzero);
    }
    if (interp2 == 1) {
        double sf = 1.0 - (double)(q0 - floorf(q0));
        double sm = 1.0 - (double)(q1 - floorf(q1));
        double sz = 1.0 - (double)(q2 - floorf(q2));
        int fs = (int)((float)C + floorf(q0));
        int ms = (int)((float)C + floorf(q1));
        int ss = (int)(floorf(q2));
        double t = val;
        add_q_to_positive_ss(h, fs, ms, ss, (uint64_t)(t * h->mult * ((sf) * (sm) * (sz))), qzero);
        add_q_to_positive_ss(h, fs + 1, ms, ss, (uint64_t)(t * h->mult * ((1 - sf) * (sm) * (sz))), qzero);
        add_q_to_positive_ss(h, fs, ms, ss + 1, (uint64_t)(t * h->mult * ((sf) * (sm) * (1 - sz))), qzero);
        add_q_to_positive_ss(h, fs + 1, ms, ss + 1, (uint64_t)(t * h->mult * ((1 - sf) * (sm) * (1 - sz))), qzero);
        add_q_to_positive_ss(h, fs, ms + 1, ss, (uint64_t)(t * h->mult * ((sf) * (1 - sm) * (sz))), qzero);
        add_q_to_positive_ss(h, fs + 1, ms + 1, ss, (uint64_t)(t * h->mult * ((1 - sf) * (1 - sm) * (sz))), qzero);
        add_q_to_positive_ss(h, fs, ms + 1, ss + 1, (uint64_t)(t * h->mult * ((sf) * (1 - sm) * (1 - sz))), qzero);
        add_q_to_positive_ss(h, fs + 1, ms + 1, ss + 1, (uint64_t)(t * h->mult * ((1 - sf) * (1 - sm) * (1 - sz))), qzero);
    }
}

static inline void rot3(const float R[9], float a, float b, float c, float out[3])
{
    out[0] = a * R[0] + b * R[1] + c * R[2];
    out[1] = a * R[3] + b * R[4] + c * R[5];
    out[2] = a * R[6] + b * R[7] + c * R[8];
}

/* Autocor_sparseHL, IAC/kernel.cl:451-652.  params follows
 * IAC/Detector.cpp:1060-1073: [0] list size, [1] Voxel_per_dq, [2] Size_AB,
 * [3] Size_C, [4] Max_Q, [5] DoubleMapping, [6] Multiplicator, [7] first-level
 * interpolation, [8] second-level interpolation.  Returns the number of
 * skipped out-of-mesh writes. */
uint64_t iaco_sparse_ac_halfmesh(const float *HL, uint32_t n_unused, const double P[9],
                                 const float R[9], uint64_t *half)
{
    (void)n_unused;
    halfmesh_t h;
    const uint32_t list = (uint32_t)P[0];
    const uint32_t dVdq = (uint32_t)P[1];
    h.ac = half;
    h.S = (int)(uint32_t)P[2];
    h.C = (h.S - 1) / 2;
    h.half_ss = (h.S + 1) / 2;
    h.mult = P[6];
    h.oob = 0;
    const float maxq = (float)P[4];
    const int dmap = (int)P[5];
    const int i1 = (int)P[7], i2 = (int)P[8];
    const int C = h.C;

#pragma omp parallel for schedule(dynamic, 4)
    for (uint32_t ind = 0; ind < list; ind++) {
        float k1[3] = {HL[4 * ind + 0], HL[4 * ind + 1], HL[4 * ind + 2]};
        double fval = (double)HL[4 * ind + 3];
        for (uint32_t i = ind; i < list; i++) {
            float q[3];
            q[0] = k1[0] - HL[4 * i + 0];
            q[1] = k1[1] - HL[4 * i + 1];
            q[2] = k1[2] - HL[4 * i + 2];
            if (i == ind) {
                add_rotated_q(&h, fval * HL[4 * i + 3], 0, 0, 0, i2, 1);
                continue;
            }
            if (sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) > maxq) continue;
            q[0] = q[0] * (float)dVdq;
            q[1] = q[1] * (float)dVdq;
            q[2] = q[2] * (float)dVdq;
            if (dmap == 1) {
                if (i1 == 0) {
                    int fs = (int)(roundf(q[0]) + (float)C);
                    int ms = (int)(roundf(q[1]) + (float)C);
                    int ss = (int)(roundf(q[2]) + (float)C);
                    float t[3];
                    rot3(R, (float)(fs - C), (float)(ms - C), (float)(ss - C), t);
                    add_rotated_q(&h, fval * HL[4 * i + 3], t[0], t[1], t[2], i2, 0);
                }
                if (i1 == 1) {
                    double sf = 1.0 - (double)(q[0] - floorf(q[0]));
                    double sm = 1.0 - (double)(q[1] - floorf(q[1]));
                    double sz = 1.0 - (double)(q[2] - floorf(q[2]));
                    int fs = (int)((float)C + floorf(q[0]));
                    int ms = (int)((float)C + floorf(q[1]));
                    int ss = (int)((float)C + floorf(q[2]));
                    float base = (float)(fval * HL[4 * i + 3]);
                    /* corner order and weights of IAC/kernel.cl:558-636 */
                    static const int cx[8] = {0, 1, 0, 1, 0, 1, 0, 1};
                    static const int cy[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                    static const int cz[8] = {0, 0, 1, 1, 0, 0, 1, 1};
                    for (int c = 0; c < 8; c++) {
                        double wx = cx[c] ? (1 - sf) : sf;
                        double wy = cy[c] ? (1 - sm) : sm;
                        double wz = cz[c] ? (1 - sz) : sz;
                        float tv = (float)(base * ((wx) * (wy) * (wz)));
                        float t[3];
                        rot3(R, (float)((fs + cx[c]) - C), (float)((ms + cy[c]) - C),
                             (float)((ss + cz[c]) - C), t);
                        add_rotated_q(&h, tv, t[0], t[1], t[2], i2, 0);
                    }
                }
            } else {
                float t[3];
                rot3(R, q[0], q[1], q[2], t);
                add_rotated_q(&h, fval * HL[4 * i + 3], t[0], t[1], t[2], i2, 0);
            }
        }
    }
    return h.oob;
}

/* Point reflection of the half mesh into the full mesh,
 * IAC/Detector.cpp:1148-1170. */
void iaco_fold_halfmesh(const uint64_t *half, uint32_t S, double mult, float step, float offset,
                        uint64_t *full)
{
    const uint32_t C = (S - 1) / 2;
#pragma omp parallel for
    for (uint32_t ss = 0; ss < (S + 1) / 2; ss++)
        for (uint32_t ms = 0; ms < S; ms++)
            for (uint32_t fs = 0; fs < S; fs++) {
                double t = (double)half[fs + (size_t)ms * S + (size_t)ss * S * S] / mult;
                uint64_t val = (uint64_t)float_to_int_d(t, step, offset);
                full[fs + (size_t)ms * S + (size_t)(ss + C) * S * S] += val;
                if (ss != 0)
                    full[(2 * C - fs) + (size_t)(2 * C - ms) * S + (size_t)(C - ss) * S * S] += val;
            }
}

/* ---- CPU route: ACMesh::Atomic_Add_q_Entry --------------------------- */

typedef struct {
    uint64_t *mesh;
    const iaco_mesh_shape *s;
    float step, offset;
    uint64_t oob;
} fullmesh_t;

static void fm_put(fullmesh_t *m, int fs, int ms, int ss, unsigned int v)
{
    const int S = (int)m->s->size_ab;
    if (fs < 0 || ms < 0 || ss < 0 || fs >= S || ms >= S || ss >= (int)m->s->size_c) {
        __atomic_fetch_add(&m->oob, 1, __ATOMIC_RELAXED);
        return;
    }
    add_u64(&m->mesh[(size_t)fs + (size_t)ms * S + (size_t)ss * S * S], v);
}

/* ACMesh::Atomic_Add_rotated_q_Entry, IAC/ACMesh.cpp:319-385 */
static void cpu_add_rotated(fullmesh_t *m, const float q[3], float value, int interp2)
{
    const iaco_mesh_shape *s = m->s;
    if (interp2 == 0) {
        int fs = (int)roundf(q[0]) + (int)s->center[0];
        int ms = (int)roundf(q[1]) + (int)s->center[1];
        int ss = (int)roundf(q[2]) + (int)s->center[2];
        unsigned int val = (unsigned int)float_to_int_f(value, m->step, m->offset);
        fm_put(m, fs, ms, ss, val);
    }
    if (interp2 == 1) {
        double sf = (double)(1 - (q[0] - floorf(q[0])));
        double sm = (double)(1 - (q[1] - floorf(q[1])));
        double sz = (double)(1 - (q[2] - floorf(q[2])));
        int fs = (int)floorf(q[0]) + (int)s->center[0];
        int ms = (int)floorf(q[1]) + (int)s->center[1];
        int ss = (int)floorf(q[2]) + (int)s->center[2];
        const float st = m->step, of = m->offset;
        fm_put(m, fs, ms, ss, (unsigned int)float_to_int_d(value * ((sf) * (sm) * (sz)), st, of));
        fm_put(m, fs + 1, ms, ss, (unsigned int)float_to_int_d(value * ((1 - sf) * (sm) * (sz)), st, of));
        fm_put(m, fs, ms, ss + 1, (unsigned int)float_to_int_d(value * ((sf) * (sm) * (1 - sz)), st, of));
        fm_put(m, fs + 1, ms, ss + 1, (unsigned int)float_to_int_d(value * ((1 - sf) * (sm) * (1 - sz)), st, of));
        fm_put(m, fs, ms + 1, ss, (unsigned int)float_to_int_d(value * ((sf) * (1 - sm) * (sz)), st, of));
        fm_put(m, fs + 1, ms + 1, ss, (unsigned int)float_to_int_d(value * ((1 - sf) * (1 - sm) * (sz)), st, of));
        fm_put(m, fs, ms + 1, ss + 1, (unsigned int)float_to_int_d(value * ((sf) * (1 - sm) * (1 - sz)), st, of));
        fm_put(m, fs + 1, ms + 1, ss + 1, (unsigned int)float_to_int_d(value * ((1 - sf) * (1 - sm) * (1 - sz)), st, of));
    }
}

/* ArrayOperators::Rotate, IAC/ArrayOperators.h:228-238 */
static inline void rotate_inplace(float v[3], const float R[9])
{
    float r[3];
    rot3(R, v[0], v[1], v[2], r);
    v[0] = r[0];
    v[1] = r[1];
    v[2] = r[2];
}

/* ACMesh::Atomic_Add_q_Entry, IAC/ACMesh.cpp:213-317 */
static void cpu_add_q(fullmesh_t *m, float q[3], const float R[9], float value, int i1, int i2,
                      int dmap)
{
    const iaco_mesh_shape *s = m->s;
    if (sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) > s->max_q) return;
    for (int d = 0; d < 3; d++) q[d] = q[d] * (float)s->voxel_per_dq;
    const int c0 = (int)s->center[0], c1 = (int)s->center[1], c2 = (int)s->center[2];
    if (dmap) {
        if (i1 == 0) {
            int fs = (int)roundf(q[0]) + c0;
            int ms = (int)roundf(q[1]) + c1;
            int ss = (int)roundf(q[2]) + c2;
            q[0] = (float)(fs - c0);
            q[1] = (float)(ms - c1);
            q[2] = (float)(ss - c2);
            rotate_inplace(q, R);
            cpu_add_rotated(m, q, value, i2);
        }
        if (i1 == 1) {
            double sf = 1.0 - (double)(q[0] - floorf(q[0]));
            double sm = 1.0 - (double)(q[1] - floorf(q[1]));
            double sz = 1.0 - (double)(q[2] - floorf(q[2]));
            int fs = (int)floorf(q[0]) + c0;
            int ms = (int)floorf(q[1]) + c1;
            int ss = (int)floorf(q[2]) + c2;
            /* corner order of IAC/ACMesh.cpp:252-306 */
            static const int cx[8] = {0, 1, 0, 1, 0, 1, 0, 1};
            static const int cy[8] = {0, 0, 0, 0, 1, 1, 1, 1};
            static const int cz[8] = {0, 0, 1, 1, 0, 0, 1, 1};
            for (int c = 0; c < 8; c++) {
                float v[3] = {(float)((fs + cx[c]) - c0), (float)((ms + cy[c]) - c1),
                              (float)((ss + cz[c]) - c2)};
                rotate_inplace(v, R);
                double wx = cx[c] ? (1 - sf) : sf;
                double wy = cy[c] ? (1 - sm) : sm;
                double wz = cz[c] ? (1 - sz) : sz;
                cpu_add_rotated(m, v, (float)(value * (wx) * (wy) * (wz)), i2);
            }
        }
    } else {
        rotate_inplace(q, R);
        cpu_add_rotated(m, q, value, i2);
    }
}

/* CPU route of Detector::AutoCorrelateSparseList, IAC/Detector.cpp:1027-1050 */
uint64_t iaco_sparse_ac_cpu_route(const float *HL, uint32_t n, const float R[9],
                                  const iaco_mesh_shape *s, int i1, int i2, int dmap,
                                  float step, float offset, uint64_t *full)
{
    fullmesh_t m = {full, s, step, offset, 0};
#pragma omp parallel for schedule(dynamic, 4)
    for (uint32_t i = 0; i < n; i++) {
        for (uint32_t j = i; j < n; j++) {
            float q[3];
            q[0] = HL[4 * i + 0] - HL[4 * j + 0];
            q[1] = HL[4 * i + 1] - HL[4 * j + 1];
            q[2] = HL[4 * i + 2] - HL[4 * j + 2];
            float val = HL[4 * i + 3] * HL[4 * j + 3];
            cpu_add_q(&m, q, R, val, i1, i2, dmap);
            q[0] = HL[4 * j + 0] - HL[4 * i + 0];
            q[1] = HL[4 * j + 1] - HL[4 * i + 1];
            q[2] = HL[4 * j + 2] - HL[4 * i + 2];
            if (i != j) cpu_add_q(&m, q, R, val, i1, i2, dmap);
        }
    }
    return m.oob;
}

/* Multiplicator of the device route, IAC/Detector.cpp:1055-1057 */
static double sparse_multiplicator(float step)
{
    double m = (double)(1.0 / step);
    if (m > 1) m = round(m);
    return m;
}

/* Detector::AutoCorrelateSparseList, IAC/Detector.cpp:1010-1181 */
int iaco_autocorrelate_sparse_list(const float *HL, uint32_t n, uint64_t det_pixels,
                                   const float R[9], const iaco_mesh_shape *s, int i1, int i2,
                                   int dmap, float step, float offset, int cpu_gpu,
                                   uint64_t *half, uint64_t *full, uint64_t *oob)
{
    float quot = ((float)n) / ((float)det_pixels);
    if (((quot < 0.01f) && (cpu_gpu == -1)) || cpu_gpu == 0) {
        uint64_t o = iaco_sparse_ac_cpu_route(HL, n, R, s, i1, i2, dmap, step, offset, full);
        if (oob) *oob += o;
        return 0;
    }
    const double mult = sparse_multiplicator(step);
    double P[9];
    P[0] = n;
    P[1] = s->voxel_per_dq;
    P[2] = s->size_ab;
    P[3] = s->size_c;
    P[4] = s->max_q;
    P[5] = (double)dmap;
    P[6] = mult;
    P[7] = i1;
    P[8] = i2;
    const size_t hn = (size_t)s->size_ab * s->size_ab * ((s->size_ab + 1) / 2);
    memset(half, 0, hn * sizeof(uint64_t));
    uint64_t o = iaco_sparse_ac_halfmesh(HL, n, P, R, half);
    if (oob) *oob += o;
    iaco_fold_halfmesh(half, s->size_ab, mult, step, offset, full);
    return 1;
}

uint64_t iaco_sparse_ac_batch(const float *HL, const uint64_t *off, uint32_t nframes,
                              const float *R, const iaco_mesh_shape *s, int i1, int i2,
                              int dmap, float step, float offset, int cpu_gpu,
                              uint64_t det_pixels, uint64_t *full)
{
    const size_t hn = (size_t)s->size_ab * s->size_ab * ((s->size_ab + 1) / 2);
    uint64_t *half = (uint64_t *)malloc(hn * sizeof(uint64_t));
    uint64_t oob = 0;
    for (uint32_t f = 0; f < nframes; f++) {
        uint32_t n = (uint32_t)(off[f + 1] - off[f]);
        iaco_autocorrelate_sparse_list(HL + 4 * off[f], n, det_pixels, R + 9 * (size_t)f, s, i1,
                                       i2, dmap, step, offset, cpu_gpu, half, full, &oob);
    }
    free(half);
    return oob;
}

/* ===================================================================== */
/* (b) dense C(q)                                                        */
/* ===================================================================== */

/* ArrayOperators::Min_Max_Mean_Value(float*), IAC/ArrayOperators.h:160-175 */
static float mean_f(const float *a, uint64_t n)
{
    double t = 0;
    for (uint64_t i = 0; i < n; i++) t += a[i];
    t = t / (double)(int)n;
    return (float)t;
}

/* Multiplicator of Detector::AutoCorrelate_CofQ_SmallMesh,
 * IAC/Detector.cpp:1211-1227 */
double iaco_cq_small_multiplicator(const float *I, uint64_t npix)
{
    float m = mean_f(I, npix);
    double mult = 1e-10;
    for (; 1 > (double)(m * m) * mult;) mult *= 10;
    return mult * 100000;
}

/* AutoCorr_CQ_small, IAC/kernel.cl:27-184, work items [row_begin, row_end).
 * Params of IAC/Detector.cpp:1230-1240 are taken from the mesh shape. */
uint64_t iaco_cq_small(const float *I, const float *K, uint64_t npix, const iaco_mesh_shape *s,
                       int interp, double mult, uint64_t r0, uint64_t r1, uint64_t *mesh)
{
    const uint32_t DetSize = (uint32_t)npix;
    const uint32_t V = s->voxel_per_dq;
    const uint32_t AB = s->size_ab, SC = s->size_c;
    const int A = (int)s->k_a, B = (int)s->k_b, Cc = (int)s->k_c;
    const float maxq = s->max_q;
    const int cab = (int)(AB - 1) / 2, cc = (int)(SC - 1) / 2;
    uint64_t oob = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : oob)
    for (uint64_t ind = r0; ind < r1; ind++) {
        float k1[3] = {K[3 * ind], K[3 * ind + 1], K[3 * ind + 2]};
        for (uint32_t i = 0; i < DetSize; i++) {
            double val = (double)(I[ind] * I[i]);
            if (val < 1e-37f) continue;
            uint64_t vc = (uint64_t)(val * mult);
            float q[3];
            q[0] = k1[0] - K[3 * i];
            q[1] = k1[1] - K[3 * i + 1];
            q[2] = k1[2] - K[3 * i + 2];
            if (sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) > maxq) continue;
            q[0] = q[0] * (float)V;
            q[1] = q[1] * (float)V;
            q[2] = q[2] * (float)V;
            if (interp == 0) {
                int fs = (int)(roundf(q[A]) + (float)cab);
                int ms = (int)(roundf(q[B]) + (float)cab);
                int ss = (int)(roundf(q[Cc]) + (float)cc);
                if (fs < 0 || ms < 0 || ss < 0 || fs >= (int)AB || ms >= (int)AB || ss >= (int)SC) {
                    oob++;
                    continue;
                }
                add_u64(&mesh[fs + (size_t)ms * AB + (size_t)ss * AB * AB], vc);
            }
            if (interp == 1) {
                double sf = (double)(1 - (q[A] - floorf(q[A])));
                double sm = (double)(1 - (q[B] - floorf(q[B])));
                double sz = (double)(1 - (q[Cc] - floorf(q[Cc])));
                int fs = (int)(floorf(q[A]) + (float)cab);
                int ms = (int)(floorf(q[B]) + (float)cab);
                int ss = (int)(floorf(q[Cc]) + (float)cc);
                static const int cx[8] = {0, 0, 1, 1, 0, 0, 1, 1};
                static const int cy[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                static const int cz[8] = {0, 1, 0, 1, 0, 1, 0, 1};
                for (int c = 0; c < 8; c++) {
                    double wx = cx[c] ? (1 - sf) : sf;
                    double wy = cy[c] ? (1 - sm) : sm;
                    double wz = cz[c] ? (1 - sz) : sz;
                    uint64_t v = (uint64_t)(val * mult * (wx * wy * wz));
                    int f = fs + cx[c], m = ms + cy[c], z = ss + cz[c];
                    if (f < 0 || m < 0 || z < 0 || f >= (int)AB || m >= (int)AB || z >= (int)SC) {
                        oob++;
                        continue;
                    }
                    add_u64(&mesh[f + (size_t)m * AB + (size_t)z * AB * AB], v);
                }
            }
        }
    }
    return oob;
}

/* Rotation/weight table and multiplicator of Detector::Merge_smallCofQ,
 * IAC/Detector.cpp:1339-1427 (the orthonormality warning is not restated). */
void iaco_cq_merge_weights(const float *R, const float *MI, uint32_t nf, const double *cq,
                           uint64_t small_n, float *rw, double *mult_out)
{
    double maxw = 0.0;
    for (uint32_t i = 0; i < nf; i++) {
        for (int d = 0; d < 9; d++) rw[10 * (size_t)i + d] = R[9 * (size_t)i + d];
        rw[10 * (size_t)i + 9] = (float)((double)MI[i] * (double)MI[i]);
        if (MI[i] > maxw) maxw = MI[i];
    }
    double t = 0;
    for (uint64_t i = 0; i < small_n; i++) t += cq[i];
    double mean_cq = t / (double)(int)small_n;
    if (!(mean_cq > 0) || !(maxw > 0)) { /* the reference's search would not end */
        *mult_out = 0;
        return;
    }
    double m = 1e-12;
    for (; 1 > maxw * maxw * mean_cq * m;) m *= 10;
    uint64_t oom = 1;
    for (; oom < nf;) oom *= 10;
    m = m / (double)oom;
    m *= 1e10;
    if (m > 0.6) m = round(m);
    if (m < 1 && m > 0.1) m = 1;
    if (m < 1e-12) m = 1e-12;
    for (uint32_t i = 0; i < nf; i++) {
        float red = (float)m;
        if (m > 0.6) red = roundf((float)m);
        float w = rw[10 * (size_t)i + 9];
        w *= red;
        w = floorf((float)((double)w + 0.5));
        rw[10 * (size_t)i + 9] = w / red;
    }
    *mult_out = m;
}

/* Merge_CQ, IAC/kernel.cl:189-344, small-mesh voxels [v0, v1).  The big mesh
 * is cubic with edge Size_AB; the slow index uses the AB centre (:287). */
uint64_t iaco_cq_merge(const double *small, const float *RW, uint32_t nf,
                       const iaco_mesh_shape *s, int interp, double mult, uint64_t v0,
                       uint64_t v1, uint64_t *big)
{
    const int AB = (int)s->size_ab, SC = (int)s->size_c;
    const int cab = (AB - 1) / 2, cc = (SC - 1) / 2;
    const uint32_t A = s->k_a, B = s->k_b, Cc = s->k_c;
    uint64_t oob = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : oob)
    for (uint64_t ind = v0; ind < v1; ind++) {
        int ss_in = (int)(ind / (uint64_t)(AB * AB));
        int ms_in = (int)((ind - (uint64_t)ss_in * AB * AB) / (uint64_t)AB);
        int fs_in = (int)(ind - (uint64_t)ss_in * AB * AB - (uint64_t)ms_in * AB);
        float qi[3] = {2, 2, 2};
        qi[A] = (float)(fs_in - cab);
        qi[B] = (float)(ms_in - cab);
        qi[Cc] = (float)(ss_in - cc);
        double vin = small[ind];
        if (vin < 1e-37f) continue;
        for (uint32_t i = 0; i < nf; i++) {
            const float *r = RW + 10 * (size_t)i;
            float qo[3];
            qo[0] = r[0] * qi[0] + r[1] * qi[1] + r[2] * qi[2];
            qo[1] = r[3] * qi[0] + r[4] * qi[1] + r[5] * qi[2];
            qo[2] = r[6] * qi[0] + r[7] * qi[1] + r[8] * qi[2];
            vin = small[ind];
            if (interp == 0) {
                vin = vin * (double)r[9] * mult;
                uint64_t vo = (uint64_t)vin;
                int fs = (int)(roundf(qo[0]) + (float)cab);
                int ms = (int)(roundf(qo[1]) + (float)cab);
                int ss = (int)(roundf(qo[2]) + (float)cab);
                if (fs < 0 || ms < 0 || ss < 0 || fs >= AB || ms >= AB || ss >= AB) {
                    oob++;
                    continue;
                }
                add_u64(&big[fs + (size_t)ms * AB + (size_t)ss * AB * AB], vo);
            }
            if (interp == 1) {
                double sf = (double)(1 - (qo[0] - floorf(qo[0])));
                double sm = (double)(1 - (qo[1] - floorf(qo[1])));
                double sz = (double)(1 - (qo[2] - floorf(qo[2])));
                int fs = (int)(floorf(qo[0]) + (float)cab);
                int ms = (int)(floorf(qo[1]) + (float)cab);
                int ss = (int)(floorf(qo[2]) + (float)cab);
                static const int cx[8] = {0, 0, 1, 1, 0, 0, 1, 1};
                static const int cy[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                static const int cz[8] = {0, 1, 0, 1, 0, 1, 0, 1};
                for (int c = 0; c < 8; c++) {
                    double wx = cx[c] ? (1 - sf) : sf;
                    double wy = cy[c] ? (1 - sm) : sm;
                    double wz = cz[c] ? (1 - sz) : sz;
                    uint64_t v = (uint64_t)(vin * mult * (double)r[9] * (wx * wy * wz));
                    int f = fs + cx[c], m = ms + cy[c], z = ss + cz[c];
                    if (f < 0 || m < 0 || z < 0 || f >= AB || m >= AB || z >= AB) {
                        oob++;
                        continue;
                    }
                    add_u64(&big[f + (size_t)m * AB + (size_t)z * AB * AB], v);
                }
            }
        }
    }
    return oob;
}

/* ===================================================================== */
/* (c) AC1D                                                              */
/* ===================================================================== */

/* Multiplicator of AC1D::Calculate_CQ, IAC/AC1D.cpp:78-91 */
double iaco_ac1d_cq_multiplicator(const float *I, uint64_t npix)
{
    float m = mean_f(I, npix);
    double mult = 1e-10;
    for (; 1 > (double)(m * m) * mult;) mult *= 10;
    mult = mult * 1e5;
    if (mult > 1e18) mult = 1e18;
    return mult;
}

/* AutoCorr_CQ_AV, IAC/kernel.cl:656-764, rows [r0, r1).  The reference
 * spreads rows over 10000 sub-histograms of ArraySize bins and the host folds
 * the flat buffer index by index modulo ArraySize (IAC/AC1D.cpp:184-192), so
 * the fold is the plain histogram with bins taken modulo ArraySize. */
uint64_t iaco_ac1d_cq(const float *I, const float *K, uint64_t npix, const iaco_ac1d_shape *s,
                      int interp, double mult, uint64_t r0, uint64_t r1, uint64_t *hist)
{
    const uint32_t DetSize = (uint32_t)npix;
    const float dq = s->dq_per_step;
    const uint32_t size = s->size;
    const float maxq = s->max_q;
    uint64_t oob = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : oob)
    for (uint64_t ind = r0; ind < r1; ind++) {
        float k1[3] = {K[3 * ind], K[3 * ind + 1], K[3 * ind + 2]};
        float Iind = I[ind];
        for (uint32_t i = 0; i < DetSize; i++) {
            double val = Iind * I[i];
            if (val < 1e-37f) continue;
            float d0 = k1[0] - K[3 * i], d1 = k1[1] - K[3 * i + 1], d2 = k1[2] - K[3 * i + 2];
            float q = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
            if (q > maxq) continue;
            q = q / dq;
            if (interp == 0) {
                long vc = (long)(val * mult);
                uint32_t sc = (uint32_t)(floor((double)q + 0.5));
                add_u64(&hist[sc % size], (uint64_t)vc);
            }
            if (interp == 1) {
                uint32_t sc1 = (uint32_t)(floorf(q));
                uint32_t sc2 = sc1 + 1;
                double sep = (double)(q - floorf(q));
                long v1 = (long)(val * (1 - sep) * mult);
                long v2 = (long)(val * (sep)*mult);
                add_u64(&hist[sc1 % size], (uint64_t)v1);
                add_u64(&hist[sc2 % size], (uint64_t)v2);
            }
        }
    }
    return oob;
}

/* VecSize of Calculate_AC_UW_Mapped, IAC/AC1D.cpp:301 */
uint32_t iaco_ac1d_vecsize(float max_q, float dqdx)
{
    return (uint32_t)((int)ceilf(max_q / dqdx) - 1);
}

/* AutoCorr_sparseHL_AAV, IAC/kernel.cl:863-950 (Multiplicator 100 and
 * MapAndReduce 10000 at IAC/AC1D.cpp:298-304), with the host fold of
 * IAC/AC1D.cpp:366-375 kept in integers: the sub-histogram stride is VecSize
 * and the fold takes flat index modulo VecSize, so a bin sc >= VecSize lands at
 * sc - VecSize.  hist has VecSize words; lists must be shorter than 10000
 * photons (the reference writes past its buffer beyond that). */
void iaco_ac1d_sparse_frame(const float *HL, uint32_t n, float max_q, float dqdx, int interp,
                            double mult, uint64_t *hist)
{
    const uint32_t vs = iaco_ac1d_vecsize(max_q, dqdx);
    for (uint32_t ind = 0; ind < n; ind++) {
        float k1[3] = {HL[4 * ind], HL[4 * ind + 1], HL[4 * ind + 2]};
        double Iind = (double)HL[4 * ind + 3];
        for (uint32_t i = 0; i < n; i++) {
            float d0 = k1[0] - HL[4 * i], d1 = k1[1] - HL[4 * i + 1], d2 = k1[2] - HL[4 * i + 2];
            float q = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
            double val = Iind * (double)HL[4 * i + 3];
            if (q > max_q) continue;
            q = q / dqdx;
            if (interp == 0) {
                uint64_t vc = (uint64_t)(val * mult);
                uint32_t sc = (uint32_t)(floor((double)q + 0.5));
                hist[sc % vs] += vc;
            }
            if (interp == 1) {
                uint32_t sc1 = (uint32_t)(floorf(q));
                uint32_t sc2 = sc1 + 1;
                double sep = (double)(q - floorf(q));
                hist[sc1 % vs] += (uint64_t)(val * (1 - sep) * mult);
                hist[sc2 % vs] += (uint64_t)(val * sep * mult);
            }
        }
    }
}

/* CPU route of Calculate_AC_UW_Mapped, IAC/AC1D.cpp:256-293 (k >= j, both
 * orientations counted by a factor 2, which also doubles the self pair). */
void iaco_ac1d_sparse_frame_cpu_route(const float *HL, uint32_t n, float max_q, float dqdx,
                                      int interp, double *ac)
{
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t k = j; k < n; k++) {
            float d0 = HL[4 * j] - HL[4 * k], d1 = HL[4 * j + 1] - HL[4 * k + 1],
                  d2 = HL[4 * j + 2] - HL[4 * k + 2];
            float q = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
            if (q > max_q) continue;
            q = q / dqdx;
            if (interp == 0) {
                uint32_t sc = (uint32_t)(floor((double)q + 0.5));
                ac[sc] += 2.0f * (HL[4 * j + 3] * HL[4 * k + 3]);
            } else {
                uint32_t sc1 = (uint32_t)(floor((double)q));
                uint32_t sc2 = sc1 + 1;
                float sep = q - (float)sc1;
                float v1 = 2.0f * ((HL[4 * j + 3] * HL[4 * k + 3]) * (1 - sep));
                float v2 = 2.0f * ((HL[4 * j + 3] * HL[4 * k + 3]) * (sep));
                ac[sc1] += v1;
                ac[sc2] += v2;
            }
        }
}

/* Calculate_AC_UW_Mapped over a list of frames, IAC/AC1D.cpp:201-391: per
 * frame the route the reference picks (route < 0: the CPU loop when
 * (float)n / (float)det_pixels < 0.0075f, :251-253; route 0: always the CPU
 * loop; route 1: always the device kernel), each adding into the double AC_M
 * of `size` bins in frame order.  The device route adds its integer totals /
 * 100 (:364-375; the reference adds each of its 10000 sub-histograms' words /
 * 100 in turn, the same doubles whenever the words are multiples of 100, as
 * they are for photon counts with nearest binning). */
void iaco_ac1d_uw_frames(const float *HL, const uint64_t *off, uint32_t nframes, uint64_t det_pixels,
                         float max_q, float dqdx, uint32_t size, int interp, int route, double *ac)
{
    const uint32_t vs = iaco_ac1d_vecsize(max_q, dqdx);
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * vs);
    for (uint32_t f = 0; f < nframes; f++) {
        const uint32_t n = (uint32_t)(off[f + 1] - off[f]);
        const float *hl = HL + 4 * off[f];
        const float quot = (float)n / (float)det_pixels;
        const int cpu = route < 0 ? (quot < 0.0075f) : (route == 0);
        if (cpu) {
            iaco_ac1d_sparse_frame_cpu_route(hl, n, max_q, dqdx, interp, ac);
        } else {
            memset(tmp, 0, sizeof(uint64_t) * vs);
            iaco_ac1d_sparse_frame(hl, n, max_q, dqdx, interp, 100.0, tmp);
            for (uint32_t j = 0; j < vs && j < size; j++) ac[j] += (double)tmp[j] / 100.0;
        }
    }
    free(tmp);
}

/* ===================================================================== */
/* (d) simulator                                                         */
/* ===================================================================== */

/* SimulateCrystal, IAC/kernel.cl:768-859.  Params of
 * IAC/Simulator.cpp:764-777: [0] emitters, [2] SubSampling, [3..5] u step,
 * [6..8] v step, [9] wavelength.  intensity_mode 0 adds |Psi| per sub-pixel
 * as the reference does (:844); 1 adds |Psi|^2. */
void iaco_simulate_crystal(const float *PM, uint64_t npix, const float *EM, uint32_t nem_unused,
                           const double P[10], int mode, float *out)
{
    (void)nem_unused;
    const double PI = 3.1415926535897932;
    const uint32_t nem = (uint32_t)P[0];
    const int susa = (int)P[2];
    const float us[3] = {(float)P[3], (float)P[4], (float)P[5]};
    const float vs[3] = {(float)P[6], (float)P[7], (float)P[8]};
    const float wl = (float)P[9];
#pragma omp parallel for schedule(static)
    for (uint64_t ind = 0; ind < npix; ind++) {
        float pc[3] = {PM[3 * ind], PM[3 * ind + 1], PM[3 * ind + 2]};
        float acc = 0.0f;
        for (int v = -susa; v <= susa; v++)
            for (int u = -susa; u <= susa; u++) {
                float re = 0, im = 0;
                float cp[3];
                for (int d = 0; d < 3; d++) cp[d] = pc[d] + ((float)v * vs[d]) + ((float)u * us[d]);
                float nk = (float)(1.0 / (double)sqrtf(cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]));
                nk = (float)((double)nk * ((2.0 * PI) / (double)wl));
                float k[3] = {cp[0] * nk, cp[1] * nk, cp[2] * nk};
                for (uint32_t i = 0; i < nem; i++) {
                    float arg = 0;
                    arg += k[0] * EM[4 * i + 0];
                    arg += k[1] * EM[4 * i + 1];
                    arg += k[2] * EM[4 * i + 2];
                    arg += EM[4 * i + 3];
                    re += cosf(arg);
                    im += sinf(arg);
                }
                if (mode == 0)
                    acc += sqrtf((re * re) + (im * im));
                else
                    acc += (re * re) + (im * im);
            }
        out[ind] = acc / ((float)((2 * susa + 1) * (2 * susa + 1)));
    }
}

/* FP64 restatement of the same sum (for error reporting). */
void iaco_simulate_crystal_f64(const float *PM, uint64_t npix, const float *EM,
                               uint32_t nem_unused, const double P[10], int mode, double *out)
{
    (void)nem_unused;
    const uint32_t nem = (uint32_t)P[0];
    const int susa = (int)P[2];
#pragma omp parallel for schedule(static)
    for (uint64_t ind = 0; ind < npix; ind++) {
        double acc = 0.0;
        for (int v = -susa; v <= susa; v++)
            for (int u = -susa; u <= susa; u++) {
                double cp[3];
                for (int d = 0; d < 3; d++)
                    cp[d] = (double)PM[3 * ind + d] + v * (double)(float)P[6 + d] +
                            u * (double)(float)P[3 + d];
                double nk = 2.0 * M_PI / (double)(float)P[9] /
                            sqrt(cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]);
                double re = 0, im = 0;
                for (uint32_t i = 0; i < nem; i++) {
                    double arg = nk * (cp[0] * EM[4 * i] + cp[1] * EM[4 * i + 1] +
                                       cp[2] * EM[4 * i + 2]) +
                                 (double)EM[4 * i + 3];
                    re += cos(arg);
                    im += sin(arg);
                }
                acc += mode == 0 ? sqrt(re * re + im * im) : re * re + im * im;
            }
        out[ind] = acc / ((2 * susa + 1) * (2 * susa + 1));
    }
}

/* Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11): ten rounds of two
 * 32x32->64 multiplies with the Weyl key schedule.  The device code in
 * incohautocorrelate_b200/csrc/rng.cuh is the same function. */
void iaco_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* Uniform double in [0, 1) with 53 random bits: draw 0 uses words 0-1 and
 * draw 1 words 2-3 of the block at counter (idx, stream), key seed. */
double iaco_uniform_double(uint64_t seed, uint64_t stream, uint64_t idx, uint32_t draw)
{
    uint32_t ctr[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), (uint32_t)stream,
                       (uint32_t)(stream >> 32)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    iaco_philox4x32_10(ctr, key, o);
    uint64_t w = draw == 0 ? (((uint64_t)o[0] << 32) | o[1]) : (((uint64_t)o[2] << 32) | o[3]);
    return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}

/* ArrayOperators::ScalarPoissonSampling, IAC/ArrayOperators.h:25-55, with the
 * global mt19937_64 replaced by the counter-based stream above.  The
 * sequential search stops once the term underflows to zero, which ends the
 * loop for a uniform draw that the rounded cumulative sum never reaches. */
uint32_t iaco_poisson(double mean, uint64_t seed, uint64_t stream, uint64_t idx)
{
    double ret = 0;
    if (mean < 25) {
        int i = 0;
        double p, q, r;
        r = exp(-mean);
        p = r;
        q = iaco_uniform_double(seed, stream, idx, 0);
        while (p < q && r > 0) {
            i++;
            r *= mean / i;
            p += r;
        }
        ret = i;
    } else {
        double u = 1 - iaco_uniform_double(seed, stream, idx, 0);
        double v = 1 - iaco_uniform_double(seed, stream, idx, 1);
        ret = (mean + sqrt(mean) * sqrt(-2. * log(u)) * cos(2. * M_PI * v));
        if (ret < 0) ret = 0;
    }
    return (uint32_t)ret;
}

void iaco_poisson_array(const float *mean, uint64_t n, uint64_t seed, uint64_t stream, float *out)
{
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; i++) out[i] = (float)iaco_poisson(mean[i], seed, stream, i);
}

/* Crystal::Create_Lattice + Create_Crystal, IAC/Crystal.cpp:192-229.
 * lattice_vec is row-major LatticeVector[3][3]; atoms gets 3 doubles per atom. */
void iaco_crystal_lattice(const double LV[9], const uint32_t cells[3], const double *uc,
                          uint32_t nuc, double *atoms)
{
    const uint32_t l = cells[0], m = cells[1], n = cells[2];
    for (uint32_t x = 0; x < l; x++)
        for (uint32_t y = 0; y < m; y++)
            for (uint32_t z = 0; z < n; z++) {
                size_t li = z + (size_t)n * y + (size_t)n * m * x;
                for (int d = 0; d < 3; d++) {
                    double p = (x - l / 2.0 + 0.5) * LV[0 * 3 + d] +
                               (y - m / 2.0 + 0.5) * LV[1 * 3 + d] +
                               (z - n / 2.0 + 0.5) * LV[2 * 3 + d];
                    for (uint32_t j = 0; j < nuc; j++) atoms[3 * (li * nuc + j) + d] = p + uc[3 * j + d];
                }
            }
}

/* Crystal::RotateVectors(angle, axis) matrix, IAC/Crystal.cpp:125-157 */
void iaco_rotation_axis_angle(double alpha, const double ax_in[3], float R[9])
{
    double N = sqrt(ax_in[0] * ax_in[0] + ax_in[1] * ax_in[1] + ax_in[2] * ax_in[2]);
    double ax[3] = {ax_in[0] / N, ax_in[1] / N, ax_in[2] / N};
    double c = cos(alpha), s = sin(alpha);
    R[0] = (float)(ax[0] * ax[0] * (1 - c) + c);
    R[1] = (float)(ax[1] * ax[0] * (1 - c) - ax[2] * s);
    R[2] = (float)(ax[2] * ax[0] * (1 - c) + ax[1] * s);
    R[3] = (float)(ax[0] * ax[1] * (1 - c) + ax[2] * s);
    R[4] = (float)(ax[1] * ax[1] * (1 - c) + c);
    R[5] = (float)(ax[2] * ax[1] * (1 - c) - ax[0] * s);
    R[6] = (float)(ax[0] * ax[2] * (1 - c) - ax[1] * s);
    R[7] = (float)(ax[1] * ax[2] * (1 - c) + ax[0] * s);
    R[8] = (float)(ax[2] * ax[2] * (1 - c) + c);
}

/* 3x3 inverse in double (the event matrix is the inverse of the crystal
 * rotation, IAC/Simulator.cpp:707-722). */
void iaco_invert3(const float m[9], float inv[9])
{
    double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
    double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    double det = a * A + b * B + c * C;
    inv[0] = (float)(A / det);
    inv[1] = (float)(-(b * i - c * h) / det);
    inv[2] = (float)((b * f - c * e) / det);
    inv[3] = (float)(B / det);
    inv[4] = (float)((a * i - c * g) / det);
    inv[5] = (float)(-(a * f - c * d) / det);
    inv[6] = (float)(C / det);
    inv[7] = (float)(-(a * h - b * g) / det);
    inv[8] = (float)((a * e - b * d) / det);
}

/* RunIAC::Merge_ACandCQ, IAC/RunIAC.cpp:120-158: AC as IntToFloat (a float,
 * IAC/Settings.h:184-187) over C(q), 0 where C(q) <= 0 or the ratio is NaN. */
void iaco_merge_ac_and_cq(const uint64_t *ac, const double *cq, uint64_t n, float step,
                          float offset, double *out)
{
    for (uint64_t i = 0; i < n; i++) {
        double a = (double)(((float)ac[i] * step) - (float)offset);
        double o = cq[i] <= 0 ? 0.0 : a / cq[i];
        if (isnan(o)) o = 0;
        out[i] = o;
    }
}
