// Detector.h + ACMesh.h -- the reference's Detector and ACMesh classes for
// the pair-correlation path, backed by libiac_b200
// (IAC/Detector.h:18-127, IAC/ACMesh.h:7-58 of FabianTr/IncohAutoCorrelate).
//
// Data members keep the reference's names and layouts ([n_y][n_x][3] pixel and
// k maps, SparseHitList of (kx, ky, kz, value), ACMesh::Mesh as uint64 S^3 in
// fs-fastest order, CQMesh as double).  The methods that ran OpenCL kernels run
// the sm_100a kernels through the C ABI.
//
// Difference in timing, not in result: AutoCorrelateSparseList enqueues the
// frame into the mesh's device batch instead of reading the mesh back after
// every frame.  The mesh on the host (ACMesh::Mesh) is brought up to date by
// ACMesh::Sync(Settings&), which RunIAC calls before it reads the mesh; set
// ACMesh::SyncEveryFrame for the reference's per-call behaviour.
#pragma once

#include <array>
#include <cstdint>
#include <vector>

#include "Settings.h"

namespace iac {

class ACMesh;

class Detector {
public:
    struct AutoCorrFlags {
        Settings::Interpolation InterpolationMode;
    };
    struct DetChecklist {
        bool SparseHitList = false, Event = false, PixelMap = false, KMap = false,
             PixelMask = false, Intensity = false;
    };
    DetChecklist Checklist;

    Detector();
    Detector(const Detector &RefDet, bool DeepCopy);
    ~Detector();
    Detector &operator=(const Detector &) = delete;

    // geometry
    void Calc_kMap();                                   // IAC/Detector.cpp:310-361
    void CreateEmptyPixelMap(int FsSize, int SsSize);   // IAC/Detector.cpp:363-374
    void LoadPixelMap(const float *pixel_map, unsigned int ss, unsigned int fs);  // array input
    void LoadPixelMask(const int *mask);                // array input (IAC/Detector.cpp:535)
    void GenerateFlatOnesPixelMask();
    void ApplyPixelMask();

    // intensities
    void LoadIntensityData(Settings::HitEvent *Event, Settings &Options);
    void LoadAndAverageIntensity(std::vector<Settings::HitEvent> &Events, float Threshold,
                                 float PhotonSamplingStep, int LowerBound, int UpperBound,
                                 bool Pixelmask, Settings &Options);  // IAC/Detector.cpp:687-790

    // sparse list (IAC/Detector.cpp:926-977)
    void CreateSparseHitList(float Threshold);
    void CreateSparseHitList(float Threshold, float PhotonSamplingStep);
    void CreateSparseHitList(float Threshold, float PhotonSamplingStep, bool Par);
    float CalculateMeanIntensity(bool FromSparse);

    // correlation (IAC/Detector.h:93-99); returns 1 (device) as the reference's GPU route
    int AutoCorrelateSparseList(ACMesh &BigMesh, AutoCorrFlags FlagsFirstMap,
                                AutoCorrFlags FlagsSecondMap, bool DoubleMapping,
                                Settings &Options, int CpuGpu = -1);
    void AutoCorrelate_CofQ_SmallMesh(ACMesh &SmallMesh, AutoCorrFlags Flags, Settings &Options);
    void Merge_smallCofQ(ACMesh &BigMesh, ACMesh &SmallMesh, std::vector<Settings::HitEvent> &Events,
                         unsigned int LowerBound, unsigned int UpperBound, Settings &Options,
                         AutoCorrFlags Flags);
    void Merge_smallCofQ(ACMesh &BigMesh, ACMesh &SmallMesh, std::vector<Settings::HitEvent> &Events,
                         Settings &Options, AutoCorrFlags Flags);

    unsigned int DetectorSize[2] = {0, 0};  // [0] slow scan (n_y), [1] fast scan (n_x)
    float *Intensity = nullptr;
    int *PixelMask = nullptr;
    float *PixelMap = nullptr;
    float *kMap = nullptr;
    float Max_k[3], Min_k[3], Max_q[3];
    std::vector<std::array<float, 4>> SparseHitList;
    Settings::HitEvent *DetectorEvent = nullptr;

    size_t Pixels() const { return (size_t)DetectorSize[0] * DetectorSize[1]; }

private:
    void alloc_arrays();
};

class ACMesh {
public:
    explicit ACMesh(Settings *PrgSettings);
    ~ACMesh();
    ACMesh(const ACMesh &) = delete;
    ACMesh &operator=(const ACMesh &) = delete;

    double *CQMesh = nullptr;
    unsigned long *Mesh = nullptr;

    struct MeshShape {
        unsigned int k_A, k_B, k_C;
        unsigned int Size_AB, Size_C;
        unsigned int Center[3];
        float dq_per_Voxel;
        unsigned int Voxel_per_dq = 1;
        float Max_Q;
    };
    MeshShape Shape;
    Settings *Options = nullptr;

    void CreateBigMeshForDetector(Detector &Det, int EdgeSize, float q_Zoom = 1.0f);
    void CreateBigMesh_CofQ_ForDetector(Detector &Det, int EdgeSize, float q_Zoom = 1.0f);
    void CreateSmallMesh_CofQ_ForDetector(Detector &Det, int PerpSize, float q_Zoom = 1.0f);

    struct ACMesh_Checklist {
        bool SmallMesh = false, BigMesh = false, CofQBigMesh = false, CofQSmallMesh = false;
    };
    ACMesh_Checklist Checklist;

    // Device batch of AutoCorrelateSparseList frames: flush pending frames,
    // fold the device half mesh and add it to Mesh.
    void Sync(Settings &Options);
    bool SyncEveryFrame = false;
    size_t PendingFrames() const { return batch_off_.size() - 1; }

    iac_mesh_shape CShape() const;

private:
    friend class Detector;
    void enqueue_frame(const std::vector<std::array<float, 4>> &list, const float rot[9],
                       const iac_sparse_params &p, Settings &Options);
    void flush(Settings &Options);
    void release_device();
    // pending frames (host) and device buffers
    std::vector<float> batch_photons_;
    std::vector<uint64_t> batch_off_{0};
    std::vector<float> batch_rot_;
    iac_sparse_params params_{};
    bool have_params_ = false;
    iac_ctx *ctx_ = nullptr;
    void *d_half_ = nullptr, *d_full_ = nullptr, *d_ph_ = nullptr, *d_off_ = nullptr, *d_rot_ = nullptr;
    size_t cap_ph_ = 0, cap_frames_ = 0;
    bool device_dirty_ = false;
};

iac_mesh_shape ToC(const ACMesh::MeshShape &s);
ACMesh::MeshShape FromC(const iac_mesh_shape &s);

}  // namespace iac
