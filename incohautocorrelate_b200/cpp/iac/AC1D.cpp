// AC1D.cpp -- angular-averaged C(q) and unweighted AC over libiac_b200
// (IAC/AC1D.cpp).
#include "AC1D.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <vector>

namespace iac {

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

AC1D::~AC1D()
{
    delete[] CQ;
    delete[] AC_UW;
    delete[] AC;
    delete[] Q;
}

void AC1D::Initialize()
{
    delete[] CQ;
    delete[] AC_UW;
    delete[] AC;
    delete[] Q;
    CQ = new double[Shape.Size]();
    AC_UW = new double[Shape.Size]();
    AC = new double[Shape.Size]();
    Q = new double[Shape.Size]();
    for (unsigned int i = 0; i < Shape.Size; i++) Q[i] = (float)i * Shape.dq_per_Step;
}

void AC1D::Initialize(Detector &Det, unsigned int ArraySize) { Initialize(Det, ArraySize, 1.0f); }

void AC1D::Initialize(Detector &Det, unsigned int ArraySize, float QZoom)
{
    iac_ac1d_shape s;
    Check(iac_ac1d_shape_init(Det.Max_q, ArraySize, QZoom, &s), "iac_ac1d_shape_init");
    Shape.Size = s.size;
    Shape.Max_Q = s.max_q;
    Shape.dq_per_Step = s.dq_per_step;
    Initialize();
}

void AC1D::Calculate_CQ(Detector &Det, Settings &Options, Settings::Interpolation Mode)
{
    iac_ctx *ctx = Options.Context();
    void *s = Options.Stream();
    const size_t n = Det.Pixels();
    double mult = 0;
    Check(iac_ac1d_cq_multiplicator(Det.Intensity, n, &mult), "AC1D multiplicator");
    const iac_ac1d_shape sh{Shape.Size, Shape.Max_Q, Shape.dq_per_Step};
    DevBuf dI(ctx, n * 4), dK(ctx, n * 12), dH(ctx, 8 * (size_t)Shape.Size);
    Check(iac_memcpy_h2d(ctx, dI.p, Det.Intensity, n * 4, s), "copy intensity");
    Check(iac_memcpy_h2d(ctx, dK.p, Det.kMap, n * 12, s), "copy k-map");
    Check(iac_memset_device(ctx, dH.p, 0, 8 * (size_t)Shape.Size, s), "clear histogram");
    Check(iac_ac1d_cq(ctx, (const float *)dI.p, (const float *)dK.p, n, &sh, Mode, mult, (uint64_t *)dH.p, s),
          "iac_ac1d_cq");
    std::vector<uint64_t> h(Shape.Size);
    Check(iac_memcpy_d2h(ctx, h.data(), dH.p, 8 * h.size(), s), "copy histogram");
    Check(iac_stream_synchronize(ctx, s), "synchronize");
    delete[] CQ;
    CQ = new double[Shape.Size]();
    // the reference divides each of its 10000 partial sums and adds the
    // quotients; the integer total divided once differs in the last bits only
    for (unsigned int j = 0; j < Shape.Size; j++) CQ[j] = (double)h[j] / mult;
}

void AC1D::Calculate_AC_UW_MR(Settings &Options, Detector &RefDet, Settings::Interpolation Mode,
                              std::array<float, 2> Ph, unsigned int Lower, unsigned int Upper, unsigned int)
{
    if (Options.HitEvents.empty() || Upper <= Lower) throw std::runtime_error("No entrys in HitEvents");
    iac_ctx *ctx = Options.Context();
    void *s = Options.Stream();
    const size_t n = RefDet.Pixels();
    const iac_ac1d_shape sh{Shape.Size, Shape.Max_Q, Shape.dq_per_Step};
    const uint64_t words = iac_ac1d_uw_words(&sh);
    DevBuf dA(ctx, 8 * (size_t)words), dU(ctx, 8 * (size_t)Shape.Size);
    Check(iac_memset_device(ctx, dA.p, 0, 8 * (size_t)words, s), "clear accumulator");
    Detector Det(RefDet, true);
    std::vector<float> photons;
    std::vector<uint64_t> off{0};
    auto flush = [&]() {
        const size_t nf = off.size() - 1;
        if (nf == 0) return;
        DevBuf dP(ctx, std::max<size_t>(photons.size(), 4) * 4), dO(ctx, 8 * off.size());
        Check(iac_memcpy_h2d(ctx, dP.p, photons.data(), photons.size() * 4, s), "copy photons");
        Check(iac_memcpy_h2d(ctx, dO.p, off.data(), 8 * off.size(), s), "copy offsets");
        // each frame takes the route the reference picks for it (IAC/AC1D.cpp:251-253)
        Check(iac_ac1d_uw_batch(ctx, (const float *)dP.p, (const uint64_t *)dO.p, (uint32_t)nf, (uint64_t)n, &sh,
                                Mode, IAC_AC1D_ROUTE_REFERENCE, (uint64_t *)dA.p, s),
              "iac_ac1d_uw_batch");
        Check(iac_stream_synchronize(ctx, s), "synchronize");
        photons.clear();
        off.assign(1, 0);
    };
    for (unsigned int i = Lower; i < Upper; i++) {
        Det.LoadIntensityData(&Options.HitEvents[i], Options);
        for (size_t j = 0; j < n; j++) Det.Intensity[j] = Det.Intensity[j] * (float)Det.PixelMask[j];
        Det.CreateSparseHitList(Ph[0], Ph[1], false);
        for (auto &e : Det.SparseHitList) photons.insert(photons.end(), e.begin(), e.end());
        off.push_back(off.back() + Det.SparseHitList.size());
        if (off.size() - 1 >= Options.SparseBatchFrames) flush();
    }
    flush();
    Check(iac_ac1d_uw_finish(ctx, (const uint64_t *)dA.p, &sh, (double *)dU.p, s), "iac_ac1d_uw_finish");
    delete[] AC_UW;
    AC_UW = new double[Shape.Size]();
    Check(iac_memcpy_d2h(ctx, AC_UW, dU.p, 8 * (size_t)Shape.Size, s), "copy AC_UW");
    Check(iac_stream_synchronize(ctx, s), "synchronize");
}

void AC1D::CalcAC()
{
    delete[] AC;
    AC = new double[Shape.Size]();
    for (unsigned int i = 0; i < Shape.Size; i++) {
        AC[i] = AC_UW[i] / CQ[i];
        if (std::isnan(AC[i])) AC[i] = 0;
    }
}

void AC1D::CreateQVector()
{
    delete[] Q;
    Q = new double[Shape.Size];
    for (unsigned int i = 0; i < Shape.Size; i++) Q[i] = i * Shape.dq_per_Step;
}

}  // namespace iac
