// AC1D.h -- angular-averaged correlation (IAC/AC1D.h of
// FabianTr/IncohAutoCorrelate) over libiac_b200.
#pragma once

#include <array>

#include "Detector.h"

namespace iac {

class AC1D {
public:
    AC1D() = default;
    ~AC1D();
    AC1D(const AC1D &) = delete;
    AC1D &operator=(const AC1D &) = delete;

    struct AC1DShape {
        unsigned int Size = 0;
        float Max_Q = 0;
        float dq_per_Step = 0;
    };
    AC1DShape Shape;

    double *CQ = nullptr;
    double *AC_UW = nullptr;
    double *AC = nullptr;
    double *Q = nullptr;
    int EchoLevel = 0;

    void Initialize();                                                  // IAC/AC1D.cpp:29-45
    void Initialize(Detector &Det, unsigned int ArraySize);             // :46-52
    void Initialize(Detector &Det, unsigned int ArraySize, float QZoom);  // :53-59

    // C(|q|) of the detector's (mean) intensity, IAC/AC1D.cpp:61-195
    void Calculate_CQ(Detector &Det, Settings &Options, Settings::Interpolation IterpolMode);
    // unweighted AC(|q|) of events [Lower, Upper) read through Options.Frames,
    // IAC/AC1D.cpp:393-469; every frame takes the route the reference picks for
    // it (IAC/AC1D.cpp:251-253), both routes run on the device; Threads is ignored
    void Calculate_AC_UW_MR(Settings &Options, Detector &RefDet, Settings::Interpolation IterpolMode,
                            std::array<float, 2> Photonisation, unsigned int LowerBoundary,
                            unsigned int UpperBoundary, unsigned int Threads = 200);
    void CalcAC();        // IAC/AC1D.cpp:482-492
    void CreateQVector();  // IAC/AC1D.cpp:472-480
};

}  // namespace iac
