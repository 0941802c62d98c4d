// Detector.cpp -- Detector and ACMesh methods of the pair-correlation path
// over libiac_b200 (IAC/Detector.cpp, IAC/ACMesh.cpp).
#include "Detector.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace iac {

// ---------------------------------------------------------------------------
// RAII device buffer on the Settings' context
// ---------------------------------------------------------------------------
namespace {
struct DevBuf {
    iac_ctx *ctx = nullptr;
    void *p = nullptr;
    DevBuf(iac_ctx *c, size_t bytes) : ctx(c) { Check(iac_device_alloc(c, bytes, &p), "iac_device_alloc"); }
    ~DevBuf()
    {
        if (p) iac_device_free(ctx, p);
    }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};
}  // namespace

iac_mesh_shape ToC(const ACMesh::MeshShape &s)
{
    iac_mesh_shape c;
    c.k_a = s.k_A;
    c.k_b = s.k_B;
    c.k_c = s.k_C;
    c.size_ab = s.Size_AB;
    c.size_c = s.Size_C;
    for (int d = 0; d < 3; d++) c.center[d] = s.Center[d];
    c.dq_per_voxel = s.dq_per_Voxel;
    c.voxel_per_dq = s.Voxel_per_dq;
    c.max_q = s.Max_Q;
    return c;
}

ACMesh::MeshShape FromC(const iac_mesh_shape &c)
{
    ACMesh::MeshShape s;
    s.k_A = c.k_a;
    s.k_B = c.k_b;
    s.k_C = c.k_c;
    s.Size_AB = c.size_ab;
    s.Size_C = c.size_c;
    for (int d = 0; d < 3; d++) s.Center[d] = c.center[d];
    s.dq_per_Voxel = c.dq_per_voxel;
    s.Voxel_per_dq = c.voxel_per_dq;
    s.Max_Q = c.max_q;
    return s;
}

// ---------------------------------------------------------------------------
// Detector
// ---------------------------------------------------------------------------
Detector::Detector() {}

Detector::Detector(const Detector &R, bool)
{
    DetectorSize[0] = R.DetectorSize[0];
    DetectorSize[1] = R.DetectorSize[1];
    Checklist = R.Checklist;
    std::memcpy(Max_k, R.Max_k, sizeof Max_k);
    std::memcpy(Min_k, R.Min_k, sizeof Min_k);
    std::memcpy(Max_q, R.Max_q, sizeof Max_q);
    alloc_arrays();
    const size_t n = Pixels();
    if (R.PixelMap) std::copy(R.PixelMap, R.PixelMap + 3 * n, PixelMap);
    if (R.kMap) std::copy(R.kMap, R.kMap + 3 * n, kMap);
    if (R.PixelMask) std::copy(R.PixelMask, R.PixelMask + n, PixelMask);
    if (R.Intensity) std::copy(R.Intensity, R.Intensity + n, Intensity);
    SparseHitList = R.SparseHitList;
    DetectorEvent = R.DetectorEvent;
}

Detector::~Detector()
{
    delete[] Intensity;
    delete[] PixelMask;
    delete[] PixelMap;
    delete[] kMap;
}

void Detector::alloc_arrays()
{
    const size_t n = Pixels();
    delete[] Intensity;
    delete[] PixelMask;
    delete[] PixelMap;
    delete[] kMap;
    Intensity = new float[n]();
    PixelMask = new int[n]();
    PixelMap = new float[3 * n]();
    kMap = new float[3 * n]();
}

// IAC/Detector.cpp:310-361 (host arithmetic, the same as iac_calc_kmap)
void Detector::Calc_kMap()
{
    for (int d = 0; d < 3; d++) {
        Max_k[d] = -100.0f;
        Min_k[d] = 100.0f;
    }
    for (size_t i = 0; i < Pixels(); i++) {
        float x = PixelMap[3 * i + 0], y = PixelMap[3 * i + 1], z = PixelMap[3 * i + 2];
        const float r = std::sqrt(x * x + y * y + z * z);
        x = x / r;
        y = y / r;
        z = z / r;
        kMap[3 * i + 0] = x;
        kMap[3 * i + 1] = y;
        kMap[3 * i + 2] = z;
        const float k[3] = {x, y, z};
        for (int d = 0; d < 3; d++) {
            if (k[d] > Max_k[d]) Max_k[d] = k[d];
            if (k[d] < Min_k[d]) Min_k[d] = k[d];
        }
    }
    for (int d = 0; d < 3; d++) Max_q[d] = std::fabs(Max_k[d] - Min_k[d]);
    Checklist.KMap = true;
}

void Detector::CreateEmptyPixelMap(int FsSize, int SsSize)
{
    DetectorSize[0] = SsSize;
    DetectorSize[1] = FsSize;
    alloc_arrays();
    Checklist.PixelMap = true;
}

void Detector::LoadPixelMap(const float *pm, unsigned int ss, unsigned int fs)
{
    DetectorSize[0] = ss;
    DetectorSize[1] = fs;
    alloc_arrays();
    std::copy(pm, pm + 3 * Pixels(), PixelMap);
    Checklist.PixelMap = true;
}

void Detector::LoadPixelMask(const int *mask)
{
    if (mask)
        std::copy(mask, mask + Pixels(), PixelMask);
    else
        std::fill(PixelMask, PixelMask + Pixels(), 1);
    Checklist.PixelMask = true;
}

void Detector::GenerateFlatOnesPixelMask() { LoadPixelMask(nullptr); }

void Detector::ApplyPixelMask()
{
    for (size_t i = 0; i < Pixels(); i++) Intensity[i] = Intensity[i] * (float)PixelMask[i];
}

void Detector::LoadIntensityData(Settings::HitEvent *Event, Settings &Options)
{
    if (!Options.Frames) throw std::runtime_error("Settings::Frames (frame source) is not set");
    Options.Frames->Load(Event->Filename, Event->Dataset, Event->Event, Intensity, Pixels());
    DetectorEvent = Event;
    Checklist.Event = true;
    Checklist.Intensity = true;
}

// IAC/Detector.cpp:687-790.  Frames are loaded on the host (FrameSource) in
// batches into pinned memory; masking, thresholding / photon discretisation,
// the per-pixel accumulation and the per-event sums run on the device
// (iac_average_frames, bit-exact with the reference).  As in the reference
// the pixel mask is always applied (a mask of ones when none was loaded).
void Detector::LoadAndAverageIntensity(std::vector<Settings::HitEvent> &Events, float Threshold,
                                       float Step, int Lower, int Upper, bool /*Pixelmask*/,
                                       Settings &Options)
{
    if (Events.empty() || Upper <= Lower) return;
    if (!Options.Frames) throw std::runtime_error("Settings::Frames (frame source) is not set");
    if (!Checklist.PixelMask) GenerateFlatOnesPixelMask();
    iac_ctx *ctx = Options.Context();
    void *s = Options.Stream();
    const size_t n = Pixels();
    const uint32_t batch = (uint32_t)std::max<size_t>(1, std::min<size_t>(64, (size_t)(256u << 20) / (4 * n)));
    void *h_frames = nullptr;
    Check(iac_host_alloc_pinned(ctx, 4 * n * batch, &h_frames), "pinned frame batch");
    struct PinnedGuard {
        iac_ctx *c;
        void *p;
        ~PinnedGuard() { iac_host_free_pinned(c, p); }
    } pin{ctx, h_frames};
    DevBuf dF(ctx, 4 * n * batch), dMask(ctx, 4 * n), dSum(ctx, 4 * n), dDiscr(ctx, 8 * n), dMean(ctx, 4 * batch),
        dPh(ctx, 4 * batch), dOut(ctx, 4 * n);
    Check(iac_memcpy_h2d(ctx, dMask.p, PixelMask, 4 * n, s), "copy mask");
    Check(iac_memset_device(ctx, dSum.p, 0, 4 * n, s), "clear sum");
    Check(iac_memset_device(ctx, dDiscr.p, 0, 8 * n, s), "clear counts");
    std::vector<float> mean(batch), ph(batch);
    float *hf = static_cast<float *>(h_frames);
    for (int i0 = Lower; i0 < Upper; i0 += (int)batch) {
        const uint32_t nb = (uint32_t)std::min<int>((int)batch, Upper - i0);
        Check(iac_stream_synchronize(ctx, s), "synchronize");  // the pinned batch is free again
        for (uint32_t k = 0; k < nb; k++)
            Options.Frames->Load(Events[i0 + k].Filename, Events[i0 + k].Dataset, Events[i0 + k].Event,
                                 hf + (size_t)k * n, n);
        Check(iac_memcpy_h2d(ctx, dF.p, hf, 4 * n * nb, s), "copy frames");
        Check(iac_average_frames(ctx, (const float *)dF.p, n, nb, (const int32_t *)dMask.p, Threshold, Step,
                                 (float *)dSum.p, (int64_t *)dDiscr.p, (float *)dMean.p, (float *)dPh.p, s),
              "iac_average_frames");
        Check(iac_memcpy_d2h(ctx, mean.data(), dMean.p, 4 * nb, s), "copy mean intensities");
        if (Step > 0) Check(iac_memcpy_d2h(ctx, ph.data(), dPh.p, 4 * nb, s), "copy photon counts");
        Check(iac_stream_synchronize(ctx, s), "synchronize");
        for (uint32_t k = 0; k < nb; k++) {
            Events[i0 + k].MeanIntensity = mean[k];
            if (Step > 0) Events[i0 + k].PhotonCount = (int)ph[k];
        }
    }
    Check(iac_average_finish(ctx, Step > 0 ? nullptr : (const float *)dSum.p,
                             Step > 0 ? (const int64_t *)dDiscr.p : nullptr, n, (uint32_t)(Upper - Lower),
                             (float *)dOut.p, s),
          "iac_average_finish");
    Check(iac_memcpy_d2h(ctx, Intensity, dOut.p, 4 * n, s), "copy intensity");
    Check(iac_stream_synchronize(ctx, s), "synchronize");
    Checklist.Intensity = true;
}

// IAC/Detector.cpp:926-977
void Detector::CreateSparseHitList(float Threshold)
{
    SparseHitList.clear();
    SparseHitList.reserve(1000);
    for (size_t i = 0; i < Pixels(); i++) {
        const float I = Intensity[i];
        if (I >= Threshold && I > 0) SparseHitList.push_back({kMap[3 * i], kMap[3 * i + 1], kMap[3 * i + 2], I});
    }
    Checklist.SparseHitList = true;
}

void Detector::CreateSparseHitList(float Threshold, float Step)
{
    CreateSparseHitList(Threshold);
    for (auto &e : SparseHitList) e[3] = std::ceil((e[3] - Threshold) / Step) * (float)(e[3] >= Threshold);
}

void Detector::CreateSparseHitList(float Threshold, float Step, bool) { CreateSparseHitList(Threshold, Step); }

float Detector::CalculateMeanIntensity(bool FromSparse)
{
    double s = 0;
    if (FromSparse)
        for (auto &e : SparseHitList) s += e[3];
    else
        for (size_t i = 0; i < Pixels(); i++) s += Intensity[i];
    s = s / (double)Pixels();
    if (DetectorEvent) DetectorEvent->MeanIntensity = (float)s;
    return (float)s;
}

// IAC/Detector.cpp:1010-1181.  The frame joins the mesh's device batch; the
// reference's route choice (CPU below 1 % hit pixels) gives the same mesh for
// photon counts, so every frame takes the device path (returns 1).
int Detector::AutoCorrelateSparseList(ACMesh &BigMesh, AutoCorrFlags F1, AutoCorrFlags F2, bool DoubleMapping,
                                      Settings &Options, int)
{
    if (!Checklist.SparseHitList) throw std::runtime_error("no sparse hit list: call CreateSparseHitList first");
    if (!Checklist.Event || !DetectorEvent) throw std::runtime_error("no event set for the detector");
    iac_sparse_params p{};
    p.shape = ToC(BigMesh.Shape);
    p.interp_first = F1.InterpolationMode;
    p.interp_second = F2.InterpolationMode;
    p.double_map = DoubleMapping ? 1 : 0;
    double m = (double)(1.0 / Options.F_I_Conversion.Step);
    if (m > 1) m = std::round(m);
    p.multiplicator = m;
    BigMesh.enqueue_frame(SparseHitList, DetectorEvent->RotMatrix, p, Options);
    if (BigMesh.SyncEveryFrame) BigMesh.Sync(Options);
    return 1;
}

// IAC/Detector.cpp:1184-1315
void Detector::AutoCorrelate_CofQ_SmallMesh(ACMesh &SmallMesh, AutoCorrFlags Flags, Settings &Options)
{
    if (!SmallMesh.Checklist.CofQSmallMesh) throw std::runtime_error("SmallMesh argument is not a CofQ-Mesh");
    iac_ctx *ctx = Options.Context();
    void *s = Options.Stream();
    const size_t n = Pixels();
    double mult = 0;
    Check(iac_cq_small_multiplicator(Intensity, n, &mult), "C(q) multiplicator");
    const iac_mesh_shape sh = ToC(SmallMesh.Shape);
    const size_t words = (size_t)sh.size_ab * sh.size_ab * sh.size_c;
    DevBuf dI(ctx, n * 4), dK(ctx, n * 12), dM(ctx, words * 8);
    Check(iac_memcpy_h2d(ctx, dI.p, Intensity, n * 4, s), "copy intensity");
    Check(iac_memcpy_h2d(ctx, dK.p, kMap, n * 12, s), "copy k-map");
    Check(iac_memset_device(ctx, dM.p, 0, words * 8, s), "clear mesh");
    Check(iac_cq_small(ctx, (const float *)dI.p, (const float *)dK.p, n, DetectorSize[1], &sh, Flags.InterpolationMode, mult,
                       (uint64_t *)dM.p, s),
          "iac_cq_small");
    std::vector<uint64_t> h(words);
    Check(iac_memcpy_d2h(ctx, h.data(), dM.p, words * 8, s), "copy mesh");
    Check(iac_stream_synchronize(ctx, s), "synchronize");
    for (size_t i = 0; i < words; i++) SmallMesh.CQMesh[i] = (double)h[i] / mult;
}

void Detector::Merge_smallCofQ(ACMesh &BigMesh, ACMesh &SmallMesh, std::vector<Settings::HitEvent> &Events,
                               Settings &Options, AutoCorrFlags Flags)
{
    Merge_smallCofQ(BigMesh, SmallMesh, Events, 0, (unsigned)Events.size(), Options, Flags);
}

// IAC/Detector.cpp:1321-1573
void Detector::Merge_smallCofQ(ACMesh &BigMesh, ACMesh &SmallMesh, std::vector<Settings::HitEvent> &Events,
                               unsigned int Lower, unsigned int Upper, Settings &Options, AutoCorrFlags Flags)
{
    if (SmallMesh.Shape.Size_AB != BigMesh.Shape.Size_AB) throw std::runtime_error("Perpendicular Mesh size does not fit");
    if (Upper > Events.size()) throw std::runtime_error("Upperbound exceeds number of Events");
    iac_ctx *ctx = Options.Context();
    void *s = Options.Stream();
    const uint32_t nf = Upper - Lower;
    std::vector<float> R(9 * (size_t)nf), MI(nf), rw(10 * (size_t)nf);
    for (uint32_t i = 0; i < nf; i++) {
        std::copy(Events[Lower + i].RotMatrix, Events[Lower + i].RotMatrix + 9, &R[9 * (size_t)i]);
        MI[i] = Events[Lower + i].MeanIntensity;
    }
    const iac_mesh_shape sh = ToC(SmallMesh.Shape);
    const size_t small_words = (size_t)sh.size_ab * sh.size_ab * sh.size_c;
    const size_t big_words = (size_t)sh.size_ab * sh.size_ab * sh.size_ab;
    double mult = 0;
    Check(iac_cq_merge_weights(R.data(), MI.data(), nf, SmallMesh.CQMesh, small_words, rw.data(), &mult),
          "merge weights");
    DevBuf dS(ctx, small_words * 8), dW(ctx, std::max<size_t>(rw.size(), 1) * 4), dB(ctx, big_words * 8);
    Check(iac_memcpy_h2d(ctx, dS.p, SmallMesh.CQMesh, small_words * 8, s), "copy small C(q)");
    Check(iac_memcpy_h2d(ctx, dW.p, rw.data(), rw.size() * 4, s), "copy weights");
    Check(iac_memset_device(ctx, dB.p, 0, big_words * 8, s), "clear mesh");
    Check(iac_cq_merge(ctx, (const double *)dS.p, (const float *)dW.p, nf, &sh, Flags.InterpolationMode, mult,
                       (uint64_t *)dB.p, s),
          "iac_cq_merge");
    std::vector<uint64_t> h(big_words);
    Check(iac_memcpy_d2h(ctx, h.data(), dB.p, big_words * 8, s), "copy mesh");
    Check(iac_stream_synchronize(ctx, s), "synchronize");
    for (size_t i = 0; i < big_words; i++) BigMesh.CQMesh[i] = (double)h[i] / mult;
}

// ---------------------------------------------------------------------------
// ACMesh
// ---------------------------------------------------------------------------
ACMesh::ACMesh(Settings *PrgSettings) : Options(PrgSettings) {}

ACMesh::~ACMesh()
{
    release_device();
    delete[] CQMesh;
    delete[] Mesh;
}

iac_mesh_shape ACMesh::CShape() const { return ToC(Shape); }

static void check_edge(int e)
{
    if (e % 2 == 0) throw std::invalid_argument("PerpSize must be odd");
}

void ACMesh::CreateBigMeshForDetector(Detector &Det, int EdgeSize, float q_Zoom)
{
    check_edge(EdgeSize);
    iac_mesh_shape c;
    Check(iac_big_mesh_shape(Det.Max_q, EdgeSize, q_Zoom, &c), "iac_big_mesh_shape");
    release_device();
    Shape = FromC(c);
    delete[] Mesh;
    Mesh = new unsigned long[(size_t)Shape.Size_AB * Shape.Size_AB * Shape.Size_C]();
    Checklist.BigMesh = true;
}

void ACMesh::CreateBigMesh_CofQ_ForDetector(Detector &Det, int EdgeSize, float q_Zoom)
{
    check_edge(EdgeSize);
    iac_mesh_shape c;
    Check(iac_big_mesh_shape(Det.Max_q, EdgeSize, q_Zoom, &c), "iac_big_mesh_shape");
    Shape = FromC(c);
    delete[] CQMesh;
    CQMesh = new double[(size_t)Shape.Size_AB * Shape.Size_AB * Shape.Size_C]();
    Checklist.CofQBigMesh = true;
}

void ACMesh::CreateSmallMesh_CofQ_ForDetector(Detector &Det, int PerpSize, float q_Zoom)
{
    check_edge(PerpSize);
    iac_mesh_shape c;
    Check(iac_small_cq_mesh_shape(Det.Max_q, PerpSize, q_Zoom, &c), "iac_small_cq_mesh_shape");
    Shape = FromC(c);
    delete[] CQMesh;
    CQMesh = new double[(size_t)Shape.Size_AB * Shape.Size_AB * Shape.Size_C]();
    Checklist.CofQSmallMesh = true;
}

void ACMesh::release_device()
{
    if (!ctx_) return;
    for (void *p : {d_half_, d_full_, d_ph_, d_off_, d_rot_})
        if (p) iac_device_free(ctx_, p);
    d_half_ = d_full_ = d_ph_ = d_off_ = d_rot_ = nullptr;
    cap_ph_ = cap_frames_ = 0;
    device_dirty_ = false;
}

void ACMesh::enqueue_frame(const std::vector<std::array<float, 4>> &list, const float rot[9],
                           const iac_sparse_params &p, Settings &Options)
{
    if (have_params_ && std::memcmp(&p, &params_, sizeof p) != 0) flush(Options);
    params_ = p;
    have_params_ = true;
    for (const auto &e : list) batch_photons_.insert(batch_photons_.end(), e.begin(), e.end());
    batch_off_.push_back(batch_off_.back() + list.size());
    batch_rot_.insert(batch_rot_.end(), rot, rot + 9);
    if (PendingFrames() >= Options.SparseBatchFrames) flush(Options);
}

void ACMesh::flush(Settings &Options)
{
    if (PendingFrames() == 0) return;
    iac_ctx *ctx = Options.Context();
    void *s = Options.Stream();
    if (ctx_ && ctx_ != ctx) release_device();
    ctx_ = ctx;
    const uint32_t S = Shape.Size_AB;
    const size_t half_b = 8 * iac_half_mesh_words(S);
    if (!d_half_) {
        Check(iac_device_alloc(ctx, half_b, &d_half_), "alloc half mesh");
        Check(iac_memset_device(ctx, d_half_, 0, half_b, s), "clear half mesh");
    }
    const size_t nph = batch_photons_.size() / 4, nf = PendingFrames();
    if (nph + 1 > cap_ph_) {
        if (d_ph_) iac_device_free(ctx, d_ph_);
        cap_ph_ = std::max<size_t>(nph + 1, 2 * cap_ph_);
        Check(iac_device_alloc(ctx, 16 * cap_ph_, &d_ph_), "alloc photons");
    }
    if (nf > cap_frames_) {
        if (d_off_) iac_device_free(ctx, d_off_);
        if (d_rot_) iac_device_free(ctx, d_rot_);
        cap_frames_ = std::max<size_t>(nf, 2 * cap_frames_);
        Check(iac_device_alloc(ctx, 8 * (cap_frames_ + 1), &d_off_), "alloc offsets");
        Check(iac_device_alloc(ctx, 36 * cap_frames_, &d_rot_), "alloc rotations");
    }
    Check(iac_memcpy_h2d(ctx, d_ph_, batch_photons_.data(), 16 * nph, s), "copy photons");
    Check(iac_memcpy_h2d(ctx, d_off_, batch_off_.data(), 8 * (nf + 1), s), "copy offsets");
    Check(iac_memcpy_h2d(ctx, d_rot_, batch_rot_.data(), 36 * nf, s), "copy rotations");
    Check(iac_sparse_ac_batch(ctx, (const float *)d_ph_, (const uint64_t *)d_off_, (const float *)d_rot_,
                              (uint32_t)nf, &params_, (uint64_t *)d_half_, s),
          "iac_sparse_ac_batch");
    // the host vectors are reused right away: wait for the copies to land
    Check(iac_stream_synchronize(ctx, s), "synchronize");
    batch_photons_.clear();
    batch_off_.assign(1, 0);
    batch_rot_.clear();
    device_dirty_ = true;
}

void ACMesh::Sync(Settings &Options)
{
    flush(Options);
    if (!device_dirty_) return;
    iac_ctx *ctx = ctx_;
    void *s = Options.Stream();
    const uint32_t S = Shape.Size_AB;
    const size_t full_b = 8 * iac_full_mesh_words(S), half_b = 8 * iac_half_mesh_words(S);
    if (!d_full_) Check(iac_device_alloc(ctx, full_b, &d_full_), "alloc full mesh");
    Check(iac_memset_device(ctx, d_full_, 0, full_b, s), "clear full mesh");
    Check(iac_sparse_fold(ctx, (const uint64_t *)d_half_, S, (uint64_t *)d_full_, s), "iac_sparse_fold");
    std::vector<uint64_t> h(iac_full_mesh_words(S));
    Check(iac_memcpy_d2h(ctx, h.data(), d_full_, full_b, s), "copy mesh");
    Check(iac_memset_device(ctx, d_half_, 0, half_b, s), "clear half mesh");
    uint64_t oob = 0;
    const iac_status st = iac_ctx_check(ctx, s, &oob);
    if (st != IAC_OK && st != IAC_ERR_OUT_OF_MESH) Check(st, "iac_ctx_check");
    if (oob) Options.Echo("WARNING: " + std::to_string(oob) + " pair writes fell outside the mesh (rotation not orthonormal?)");
    for (size_t i = 0; i < h.size(); i++) Mesh[i] += h[i];
    device_dirty_ = false;
}

}  // namespace iac
