// Settings.h -- the reference's Settings class for the pair-correlation path,
// backed by libiac_b200 (IAC/Settings.h:105-187 of FabianTr/IncohAutoCorrelate).
//
// Kept: HitEvent (row-major RotMatrix, q = M * q_local), the Interpolation
// enum, F_I_Conversion with FloatToInt / IntToFloat, the HitEvents list with
// its XML file format, Echo.  SetUp_OpenCL creates the CUDA context instead of
// the OpenCL device pool (IAC/Settings.cpp:331-470); the pool's busy-wait is
// gone because every method enqueues on the context's stream.
#pragma once

#include <array>
#include <cmath>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "iac_b200.h"

namespace iac {

// Where frame intensities come from.  The reference reads HDF5 slices per
// HitEvent (IAC/Detector.cpp:136-230, :793-831); this build keeps that
// interface abstract and ships a raw-binary reader (RawStackSource) and an
// in-memory source (MemoryFrameSource).
class FrameSource {
public:
    virtual ~FrameSource() = default;
    // fill `intensity` (npix floats) with the frame the event points to
    virtual void Load(const std::string &filename, const std::string &dataset, int event,
                      float *intensity, size_t npix) = 0;
};

class Settings {
public:
    const static int XML_HITLIST_VERSION = 9;

    Settings();
    ~Settings();
    Settings(const Settings &) = delete;
    Settings &operator=(const Settings &) = delete;

    struct HitEvent {
        float RotMatrix[9];  // ROW MAJOR: q = M * q_local
        std::string Filename;
        std::string Dataset;
        int Event = 0;
        int SerialNumber = 0;
        float MeanIntensity = -1.0f;
        int PhotonCount = -1;
        float HitsPixelRatio = -1.0f;
        std::string SupplementInfo = "";
    };
    std::vector<HitEvent> HitEvents;

    bool echo = true;
    void Echo(std::string output);

    // device set-up (replaces the OpenCL platform/device pool)
    void SetUp_OpenCL();            // name kept for callers; creates the context on device 0
    void SetUp_Device(int device);  // explicit device
    iac_ctx *Context();             // created on first use
    void *Stream();                 // the stream every method enqueues on

    // event list (XML, IAC/Settings.cpp:473-676), versions 1 and >= 2
    void SafeHitEventListToFile(std::string Filename);
    void SafeHitEventListToFile(std::string Filename, std::vector<HitEvent> &List,
                                bool AdditionalInformations = false,
                                std::unordered_map<std::string, std::string> AdditioInfoMap = {});
    void LoadHitEventListFromFile(std::string Filename);
    void InvertRotationMatrices();

    enum Interpolation { NearestNeighbour = 0, Linear = 1 };

    struct FloatIntConversion {
        float Offset = 0.0f;
        float Step = 0.001f;
    };
    FloatIntConversion F_I_Conversion;
    inline long FloatToInt(float f)
    {
        return (long)floorf(((f + F_I_Conversion.Offset) / F_I_Conversion.Step) + 0.5f);
    }
    inline long FloatToInt(double f)
    {
        return (long)std::floor(((f + F_I_Conversion.Offset) / F_I_Conversion.Step) + 0.5);
    }
    inline float IntToFloat(int i) { return ((float)i * F_I_Conversion.Step) - (float)F_I_Conversion.Offset; }
    inline float IntToFloat(long i) { return ((float)i * F_I_Conversion.Step) - (float)F_I_Conversion.Offset; }
    inline float IntToFloat(unsigned long i)
    {
        return ((float)i * F_I_Conversion.Step) - (float)F_I_Conversion.Offset;
    }

    // frame input used by LoadIntensityData / Calculate_AC_UW_MR / averaging
    std::shared_ptr<FrameSource> Frames;

    // Frames handed to the batched sparse correlator per device launch.
    unsigned int SparseBatchFrames = 8192;

private:
    iac_ctx *ctx_ = nullptr;
    void *stream_ = nullptr;
    int device_ = 0;
};

// Throws std::runtime_error with iac_last_error() on a failed call.
void Check(iac_status st, const char *what);

// Raw float32 stacks: Filename names a file of [frames][npix] float32;
// Event is the frame index.  Dataset is ignored.
class RawStackSource : public FrameSource {
public:
    void Load(const std::string &filename, const std::string &dataset, int event, float *intensity,
              size_t npix) override;
};

// Frames held in memory, addressed by Event (Filename/Dataset ignored).
class MemoryFrameSource : public FrameSource {
public:
    std::vector<std::vector<float>> Frames;
    void Load(const std::string &filename, const std::string &dataset, int event, float *intensity,
              size_t npix) override;
};

}  // namespace iac
