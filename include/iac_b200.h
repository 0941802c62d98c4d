/*
 * iac_b200.h -- C ABI of libiac_b200.so, the B200 (sm_100a) implementation of
 * IncohAutoCorrelate's pair-correlation path.
 *
 * Plain C: pointers, sizes, status codes.  Device pointers ("d_") are CUDA
 * global-memory addresses on the context's device; host pointers ("h_") are
 * ordinary (preferably pinned) host memory.  `stream` is a cudaStream_t passed
 * as void* (NULL = the legacy default stream).  Every function returns an
 * iac_status; a non-IAC_OK return leaves a message for iac_last_error().
 *
 * Each entry point names the reference interface it replaces
 * (FabianTr/IncohAutoCorrelate, IncohAutoCorrelate/ abbreviated IAC/).
 * Mesh layouts are the reference's: voxel (fs, ms, ss) at fs + ms*S + ss*S*S,
 * fs running fastest, centre C = (S-1)/2 (IAC/ACMesh.cpp:84-105).
 */
#ifndef IAC_B200_H
#define IAC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IAC_ABI_VERSION 1

typedef enum {
    IAC_OK = 0,
    IAC_ERR_INVALID_ARG = 1,  /* bad size, even mesh edge, null pointer, ... */
    IAC_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    IAC_ERR_NO_MEMORY = 3,    /* device or pinned allocation failed */
    IAC_ERR_TIMEOUT = 4,      /* a bounded device-side wait ran out */
    IAC_ERR_OUT_OF_MESH = 5,  /* writes fell outside the mesh and were skipped */
    IAC_ERR_UNSUPPORTED = 6   /* no sm_100 device, or a mode not built */
} iac_status;

/* Settings::Interpolation, IAC/Settings.h:158 */
typedef enum { IAC_NEAREST = 0, IAC_LINEAR = 1 } iac_interpolation;

/* ACMesh::MeshShape, IAC/ACMesh.h:21-29 */
typedef struct {
    uint32_t k_a, k_b, k_c;    /* q axis on the fast / medium / slow mesh axis */
    uint32_t size_ab, size_c;  /* edge lengths including the 2-voxel padding */
    uint32_t center[3];
    float dq_per_voxel;
    uint32_t voxel_per_dq;
    float max_q;
} iac_mesh_shape;

/* AC1D::Shape, IAC/AC1D.h */
typedef struct {
    uint32_t size;
    float max_q;
    float dq_per_step;
} iac_ac1d_shape;

typedef struct iac_ctx iac_ctx;

/* ---------------------------------------------------------------------- */
/* context, errors                                                          */
/* ---------------------------------------------------------------------- */

/* Replaces Settings::SetUp_OpenCL + the OCL device pool
 * (IAC/Settings.cpp:331-470).  One context per device; thread-safe; calls
 * from several host threads may share it, each on its own stream. */
iac_status iac_ctx_create(int device, iac_ctx **out);
iac_status iac_ctx_destroy(iac_ctx *ctx);
/* Synchronises `stream`, then reports and clears the context's device-side
 * error counters: writes skipped because their voxel lay outside the mesh
 * (the reference writes them out of bounds; IAC_ERR_OUT_OF_MESH), photons
 * dropped because a photon list was full (IAC_ERR_NO_MEMORY) and bounded
 * waits that ran out (IAC_ERR_TIMEOUT).  The counters are shared by all of
 * the context's streams but only `stream` is waited for: work still running on
 * another stream may count after the read, and its counts are then cleared
 * with the others -- synchronise those streams first. */
iac_status iac_ctx_check(iac_ctx *ctx, void *stream, uint64_t *out_of_mesh);
const char *iac_status_string(iac_status s);
const char *iac_last_error(void); /* thread-local message of the last failure */
int iac_abi_version(void);
/* Failure paths without a GPU fault (the reference has no error recovery: its
 * device-pool wait has no timeout, IAC/Detector.cpp:1078-1081).
 * iac_ctx_set_scratch_limit: the largest device scratch buffer the context may
 * grow (0: no limit); a call that needs more fails with IAC_ERR_NO_MEMORY before
 * allocating, which both caps the library's working memory and lets callers
 * test their out-of-memory handling.
 * iac_ctx_wait_flag: one device thread waits for *d_flag != 0, at most
 * max_polls polls of about 1 us (<= 10^7); a wait that runs out is counted and
 * the next iac_ctx_check returns IAC_ERR_TIMEOUT, the context staying usable:
 * the error path every bounded wait of the library's kernels takes. */
iac_status iac_ctx_set_scratch_limit(iac_ctx *ctx, uint64_t max_bytes);
iac_status iac_ctx_wait_flag(iac_ctx *ctx, const uint32_t *d_flag, uint32_t max_polls, void *stream);
/* number of launches of this library's kernels since the context was made */
uint64_t iac_ctx_launch_count(const iac_ctx *ctx);

/* ---------------------------------------------------------------------- */
/* memory and streams (so that FFI callers need not link the CUDA runtime)  */
/* ---------------------------------------------------------------------- */

iac_status iac_device_alloc(iac_ctx *ctx, size_t bytes, void **d_ptr);
iac_status iac_device_free(iac_ctx *ctx, void *d_ptr);
iac_status iac_host_alloc_pinned(iac_ctx *ctx, size_t bytes, void **h_ptr);
iac_status iac_host_free_pinned(iac_ctx *ctx, void *h_ptr);
iac_status iac_memcpy_h2d(iac_ctx *ctx, void *d_dst, const void *h_src, size_t bytes, void *stream);
iac_status iac_memcpy_d2h(iac_ctx *ctx, void *h_dst, const void *d_src, size_t bytes, void *stream);
iac_status iac_memcpy_d2d(iac_ctx *ctx, void *d_dst, const void *d_src, size_t bytes, void *stream);
iac_status iac_memset_device(iac_ctx *ctx, void *d_ptr, int value, size_t bytes, void *stream);
iac_status iac_stream_create(iac_ctx *ctx, void **stream);
iac_status iac_stream_destroy(iac_ctx *ctx, void *stream);
iac_status iac_stream_synchronize(iac_ctx *ctx, void *stream);

/* ---------------------------------------------------------------------- */
/* geometry (host arithmetic, no device work)                               */
/* ---------------------------------------------------------------------- */

/* Detector::Calc_kMap, IAC/Detector.cpp:310-361 (k-map on the device:
 * d_kmap = d_pixel_map / |d_pixel_map|; max_q[3] returned to the host). */
iac_status iac_calc_kmap(iac_ctx *ctx, const float *d_pixel_map, uint64_t npix, float *d_kmap,
                         float max_q[3], void *stream);
/* ACMesh::CreateBigMeshForDetector, IAC/ACMesh.cpp:74-106 */
iac_status iac_big_mesh_shape(const float max_q[3], int edge_size, float q_zoom,
                              iac_mesh_shape *shape);
/* ACMesh::CreateSmallMesh_CofQ_ForDetector, IAC/ACMesh.cpp:140-206 */
iac_status iac_small_cq_mesh_shape(const float max_q[3], int perp_size, float q_zoom,
                                   iac_mesh_shape *shape);
/* AC1D::Initialize(Det, ArraySize, QZoom), IAC/AC1D.cpp:53-59 */
iac_status iac_ac1d_shape_init(const float max_q[3], uint32_t array_size, float q_zoom,
                               iac_ac1d_shape *shape);

/* ---------------------------------------------------------------------- */
/* (a) sparse photon pairs -> uint64 3D q-mesh                              */
/* ---------------------------------------------------------------------- */

/* Options of Detector::AutoCorrelateSparseList (IAC/Detector.h:93). */
typedef struct {
    iac_mesh_shape shape;   /* big cubic mesh, CreateBigMeshForDetector */
    int32_t interp_first;   /* FlagsFirstMap.InterpolationMode  */
    int32_t interp_second;  /* FlagsSecondMap.InterpolationMode */
    int32_t double_map;     /* DoubleMapping                    */
    double multiplicator;   /* round(1/F_I_Conversion.Step) = 1000, IAC/Detector.cpp:1055-1057 */
} iac_sparse_params;

/* Number of uint64 words of the half mesh S*S*((S+1)/2) and full mesh S^3. */
uint64_t iac_half_mesh_words(uint32_t size_ab);
uint64_t iac_full_mesh_words(uint32_t size_ab);

/* Batched device route of Detector::AutoCorrelateSparseList
 * (IAC/Detector.cpp:1053-1146 + kernel Autocor_sparseHL, IAC/kernel.cl:451-652)
 * for nframes frames at once.
 *   d_photons       float4 (kx, ky, kz, count) per photon, frames concatenated
 *                   (the SparseHitList layout, IAC/Detector.h:120)
 *   d_frame_offsets nframes+1 photon offsets (uint64)
 *   d_rot9          9 floats per frame, row-major HitEvent::RotMatrix
 *                   (IAC/Settings.h:107)
 *   d_half_mesh     accumulates the half mesh (ss >= 0) of the reference
 *                   kernel, uint64[iac_half_mesh_words(S)]; not cleared.
 * The call is asynchronous on `stream`.  It uses the context's scratch
 * (work-queue counters and the per-frame tile table). */
iac_status iac_sparse_ac_batch(iac_ctx *ctx, const float *d_photons,
                               const uint64_t *d_frame_offsets, const float *d_rot9,
                               uint32_t nframes, const iac_sparse_params *params,
                               uint64_t *d_half_mesh, void *stream);

/* Point reflection of the half mesh into the full mesh, the fold of
 * IAC/Detector.cpp:1147-1170 (d_full += mirror(d_half)).  The reference folds
 * after every frame through FloatToInt(half/Multiplicator); that map is the
 * identity while a frame adds less than 1.05e7 to one half-mesh voxel, so one
 * fold per batch gives the same mesh (see iac_sparse_ac_frames_host). */
iac_status iac_sparse_fold(iac_ctx *ctx, const uint64_t *d_half_mesh, uint32_t size_ab,
                           uint64_t *d_full_mesh, void *stream);

/* End-to-end replacement for a loop of Detector::AutoCorrelateSparseList
 * calls on host data (RunIAC per-frame loop, IAC/RunIAC.cpp:524-550):
 * host photon lists in, h_full_mesh (uint64[S^3], ACMesh::Mesh layout)
 * accumulated (+=) on return.  Synchronous. */
iac_status iac_sparse_ac_frames_host(iac_ctx *ctx, const float *h_photons,
                                     const uint64_t *h_frame_offsets, const float *h_rot9,
                                     uint32_t nframes, const iac_sparse_params *params,
                                     uint64_t *h_full_mesh);

/* Host photon lists binned into a device half mesh that the caller keeps
 * resident across calls (no counterpart call in the reference, whose ACMesh
 * lives on the host and is read back after every frame,
 * IAC/Detector.cpp:1100-1170): a run of many batches pays the mesh transfer
 * once, at its end (iac_sparse_fold + one copy), instead of per batch as
 * iac_sparse_ac_frames_host does.  d_half (uint64[iac_half_mesh_words(S)])
 * accumulates; the frames are copied in chunks that overlap the binning on
 * `stream`.  Returns once the host buffers have been read; the binning
 * continues on `stream`.  Calls on one context are serialised. */
iac_status iac_sparse_ac_frames_host_to_device(iac_ctx *ctx, const float *h_photons,
                                               const uint64_t *h_frame_offsets, const float *h_rot9,
                                               uint32_t nframes, const iac_sparse_params *params,
                                               uint64_t *d_half_mesh, void *stream);

/* Allocation-free form of iac_sparse_ac_batch (no counterpart in the
 * reference, which creates OpenCL buffers on every call).  For callers that
 * may not allocate device memory while they run -- an acquisition loop that
 * cannot take the synchronisation and latency of cudaMalloc/cudaFree, or a
 * host framework that owns all device memory -- this call keeps its work
 * queue in a fixed 1.8 MB array of device memory inside the library (present
 * on every GPU that loads it, until the process exits) and calls no
 * allocator.  Same arguments and result as iac_sparse_ac_batch, at most
 * 200 000 frames per call (more is rejected with IAC_ERR_INVALID_ARG).
 * iac_ctx_create looks up the array's device address on the context's device
 * (a step that may load the library's device code there); the call itself
 * only uses the address the context keeps.  Calls share the array: two calls
 * that run on the GPU at the same time (on different streams) race, so keep
 * them on one stream or otherwise ordered. */
iac_status iac_sparse_ac_batch_static(iac_ctx *ctx, const float *d_photons,
                                      const uint64_t *d_frame_offsets, const float *d_rot9,
                                      uint32_t nframes, const iac_sparse_params *params,
                                      uint64_t *d_half_mesh, void *stream);

/* Work-queue tuning of the persistent pair kernel.  Fields left 0 come from
 * the autotuner's table (tuning/sparse_tuning.tsv beside the library, or the
 * file named by IAC_SPARSE_TUNING; the row of the nearest mesh edge), else
 * from built-in defaults.  iac_sparse_get_tuning reports the setting a batch
 * on a mesh of edge size_ab would use. */
typedef struct {
    uint32_t tile_pairs;      /* pairs per queue tile           */
    uint32_t block_threads;   /* threads per CTA                */
    uint32_t ctas_per_sm;     /* persistent CTAs per SM         */
    uint32_t cache_hints;     /* L2 policy: 1 = keep the mesh resident (evict-last
                                 atomics, evict-first photon loads), 2 = none  */
} iac_sparse_tuning;
iac_status iac_sparse_set_tuning(iac_ctx *ctx, const iac_sparse_tuning *t);
iac_status iac_sparse_get_tuning(iac_ctx *ctx, uint32_t size_ab, iac_sparse_tuning *t);

/* ---------------------------------------------------------------------- */
/* (b) dense mean-intensity C(q)                                            */
/* ---------------------------------------------------------------------- */

/* Multiplicator of Detector::AutoCorrelate_CofQ_SmallMesh
 * (IAC/Detector.cpp:1211-1227): 10^k * 1e5 with Mean(I)^2 * 10^k >= 1.
 * Host arithmetic on a host array. */
iac_status iac_cq_small_multiplicator(const float *h_intensity, uint64_t npix, double *mult);

/* Kernel AutoCorr_CQ_small (IAC/kernel.cl:27-184) of
 * Detector::AutoCorrelate_CofQ_SmallMesh (IAC/Detector.cpp:1184-1315): every
 * ordered pixel pair of the mean intensity, (uint64)(I_a*I_b*Mult) binned at
 * q = k_a - k_b on the small mesh (nearest or 8-corner linear).
 * d_mesh (uint64[size_ab^2 * size_c], CQMesh order) is accumulated, not
 * cleared; CQMesh = d_mesh / Mult.  fast_size is the detector row length
 * (DetectorSize[1]); given, the kernel works on 16 x 16 pixel patches whose
 * pair differences stay within a small shared-memory window (0 = unknown
 * pixel order).  Asynchronous on `stream`. */
iac_status iac_cq_small(iac_ctx *ctx, const float *d_intensity, const float *d_kmap,
                        uint64_t npix, uint32_t fast_size, const iac_mesh_shape *small_shape,
                        int interp, double multiplicator, uint64_t *d_mesh, void *stream);

/* One share of iac_cq_small for a run on several GPUs (the reference runs the
 * kernel of IAC/kernel.cl:27-184 on one device): the unordered tile pairs are
 * dealt round-robin over `nparts` shares and this call bins share `part` into
 * d_mesh (accumulated).  The shares' meshes summed (one integer reduction,
 * e.g. an NCCL sum of the uint64 meshes) equal iac_cq_small bit for bit, for
 * any nparts; dealing the tile pairs round-robin spreads near and far (culled)
 * pairs evenly.  part < nparts.  Asynchronous. */
iac_status iac_cq_small_part(iac_ctx *ctx, const float *d_intensity, const float *d_kmap,
                             uint64_t npix, uint32_t fast_size, const iac_mesh_shape *small_shape,
                             int interp, double multiplicator, uint32_t part, uint32_t nparts,
                             uint64_t *d_mesh, void *stream);

/* The work items `ind` = d_rows[0 .. nrows) of AutoCorr_CQ_small
 * (IAC/kernel.cl:27-184): for each listed pixel ind and every pixel i, the
 * ordered pair (ind, i) binned exactly as that work item does, accumulated into
 * d_mesh (no reflection; the mesh is the sum of these items over every ind,
 * which iac_cq_small computes pair-symmetrically).  For checking a full-size
 * detector against the oracle on a subset of rows.  Row indices >= npix are
 * counted (iac_ctx_check, IAC_ERR_OUT_OF_MESH) and skipped.  nrows <= 16 776 960.
 * Asynchronous. */
iac_status iac_cq_small_rows(iac_ctx *ctx, const float *d_intensity, const float *d_kmap, uint64_t npix,
                             const uint32_t *d_rows, uint32_t nrows, const iac_mesh_shape *small_shape,
                             int interp, double multiplicator, uint64_t *d_mesh, void *stream);

/* Rotation/weight table and Multiplicator of Detector::Merge_smallCofQ
 * (IAC/Detector.cpp:1339-1427): h_rw10 gets 9 rotation floats + the rounded
 * weight MeanIntensity^2 per frame.  Host arithmetic. */
iac_status iac_cq_merge_weights(const float *h_rot9, const float *h_mean_intensity,
                                uint32_t nframes, const double *h_small_cq, uint64_t small_words,
                                float *h_rw10, double *mult);

/* Kernel Merge_CQ (IAC/kernel.cl:189-344): every small-mesh voxel with
 * C >= 1e-37 rotated by every frame's matrix and added, weighted, to the
 * cubic mesh d_big (uint64[size_ab^3]), which is accumulated, not cleared;
 * CQMesh(big) = d_big / Mult.  Asynchronous. */
iac_status iac_cq_merge(iac_ctx *ctx, const double *d_small_cq, const float *d_rw10,
                        uint32_t nframes, const iac_mesh_shape *small_shape, int interp,
                        double multiplicator, uint64_t *d_big, void *stream);

/* ---------------------------------------------------------------------- */
/* (c) AC1D                                                                 */
/* ---------------------------------------------------------------------- */

/* Multiplicator of AC1D::Calculate_CQ (IAC/AC1D.cpp:78-91). Host. */
iac_status iac_ac1d_cq_multiplicator(const float *h_intensity, uint64_t npix, double *mult);

/* Kernel AutoCorr_CQ_AV (IAC/kernel.cl:656-764) of AC1D::Calculate_CQ
 * (IAC/AC1D.cpp:61-195): |q| histogram of all ordered pixel pairs of the mean
 * intensity into d_hist (uint64[shape.size], accumulated).  Equals the sum of
 * the reference's 10000 sub-histograms; CQ = d_hist / Mult.  Asynchronous. */
iac_status iac_ac1d_cq(iac_ctx *ctx, const float *d_intensity, const float *d_kmap,
                       uint64_t npix, const iac_ac1d_shape *shape, int interp,
                       double multiplicator, uint64_t *d_hist, void *stream);

/* One share of iac_ac1d_cq (kernel AutoCorr_CQ_AV, IAC/kernel.cl:656-764) for
 * a run on several GPUs, dealt as iac_cq_small_part deals its tile pairs; the
 * shares' histograms summed equal iac_ac1d_cq bit for bit.  Asynchronous. */
iac_status iac_ac1d_cq_part(iac_ctx *ctx, const float *d_intensity, const float *d_kmap,
                            uint64_t npix, const iac_ac1d_shape *shape, int interp,
                            double multiplicator, uint32_t part, uint32_t nparts, uint64_t *d_hist,
                            void *stream);

/* The work items `ind` = d_rows[0 .. nrows) of AutoCorr_CQ_AV
 * (IAC/kernel.cl:656-764) into d_hist (uint64[shape.size], accumulated), each
 * ordered pair (ind, i) binned exactly as that work item does (bins modulo
 * Size, the sub-histogram fold).  Summed over every ind it equals iac_ac1d_cq.
 * Asynchronous. */
iac_status iac_ac1d_cq_rows(iac_ctx *ctx, const float *d_intensity, const float *d_kmap, uint64_t npix,
                            const uint32_t *d_rows, uint32_t nrows, const iac_ac1d_shape *shape, int interp,
                            double multiplicator, uint64_t *d_hist, void *stream);

/* VecSize = ceil(MaxQ / dq) - 1 of Calculate_AC_UW_Mapped (IAC/AC1D.cpp:301). */
uint32_t iac_ac1d_vecsize(float max_q, float dqdx);

/* Kernel AutoCorr_sparseHL_AAV (IAC/kernel.cl:863-950) over a batch of
 * photon lists (layout as iac_sparse_ac_batch), the device route of
 * Calculate_AC_UW_Mapped (IAC/AC1D.cpp:295-379): every ordered pair of each
 * frame, self pairs included, into d_hist (uint64[iac_ac1d_vecsize], bins
 * taken modulo VecSize as the reference's fold does; accumulated).
 * AC_UW = d_hist / Mult (Mult = 100 in the reference).  Asynchronous. */
iac_status iac_ac1d_sparse_batch(iac_ctx *ctx, const float *d_photons,
                                 const uint64_t *d_frame_offsets, uint32_t nframes, float max_q,
                                 float dqdx, int interp, double multiplicator, uint64_t *d_hist,
                                 void *stream);

/* Route of a frame in iac_ac1d_uw_batch. */
#define IAC_AC1D_ROUTE_REFERENCE (-1) /* per frame, as IAC/AC1D.cpp:251-253 decides */
#define IAC_AC1D_ROUTE_HOST 0         /* the reference's CPU loop (IAC/AC1D.cpp:254-293) */
#define IAC_AC1D_ROUTE_DEVICE 1       /* AutoCorr_sparseHL_AAV (IAC/AC1D.cpp:295-379) */

/* Words (uint64) of the accumulator of iac_ac1d_uw_batch: VecSize + 2 * Size. */
uint64_t iac_ac1d_uw_words(const iac_ac1d_shape *shape);

/* Both routes of Calculate_AC_UW_Mapped (IAC/AC1D.cpp:201-391) for a batch of
 * photon lists (layout as iac_sparse_ac_batch).  With route
 * IAC_AC1D_ROUTE_REFERENCE each frame takes the route the reference picks:
 * the CPU loop when (float)n / (float)detector_pixels < 0.0075f, which counts
 * every unordered pair k >= j with a factor 2 in float (self pair included:
 * 2 v^2 at bin 0) into Size bins, else the device kernel (every ordered pair,
 * Multiplicator 100, bins modulo VecSize).  d_acc (uint64[iac_ac1d_uw_words],
 * zeroed before the first batch, then accumulated) holds both routes' sums;
 * iac_ac1d_uw_finish turns it into AC_UW.  For photon counts with nearest
 * binning AC_UW equals the reference's bit for bit; linear binning sums
 * fractional floats in double, equal to the reference's up to the order of
 * the double additions.  VecSize + 2 Size <= 24576.  Asynchronous. */
iac_status iac_ac1d_uw_batch(iac_ctx *ctx, const float *d_photons, const uint64_t *d_frame_offsets,
                             uint32_t nframes, uint64_t detector_pixels, const iac_ac1d_shape *shape,
                             int interp, int route, uint64_t *d_acc, void *stream);
/* AC_UW (double[Size]) from the accumulator: device-route sums / 100 plus
 * the host-route sums (IAC/AC1D.cpp:366-375 and :263-292).  Asynchronous. */
iac_status iac_ac1d_uw_finish(iac_ctx *ctx, const uint64_t *d_acc, const iac_ac1d_shape *shape,
                              double *d_ac_uw, void *stream);

/* ---------------------------------------------------------------------- */
/* (d) simulator                                                            */
/* ---------------------------------------------------------------------- */

/* Crystal::EmittingCrystSettings (IAC/Crystal.h:37-44) */
typedef struct {
    int32_t incoherent;          /* random phase per emitter and mode       */
    float fluorescence_yield;    /* 0 < FlYield <= 1                        */
    int32_t random_orientation;  /* roll an orientation per frame           */
    float isotropy;              /* 0 <= Isotropie <= 1                     */
} iac_crystal_params;

/* Crystal::GetEmitters for every (frame, mode) (IAC/Crystal.cpp:29-120, with
 * the rotation stored inverted as IAC/Simulator.cpp:707-722 does).
 *   d_atoms      3 doubles per atom (Crystal::AtomPositions)
 *   d_emitters   float4 (x, y, z, phase), [frame][mode][atom]; the first
 *                d_em_count[frame*nmodes + mode] entries of each block are used
 *   d_rot_event  9 floats per frame (HitEvent::RotMatrix, the inverse)
 *   d_rot_crystal optional, 9 floats per frame (the crystal rotation)
 * Random numbers: Philox4x32-10 streams keyed by `seed`, a pure function of
 * (frame, mode, atom).  Asynchronous. */
iac_status iac_crystal_emitters(iac_ctx *ctx, const double *d_atoms, uint32_t natoms,
                                uint32_t nframes, uint32_t nmodes, const iac_crystal_params *cp,
                                uint64_t seed, float *d_emitters, uint32_t *d_em_count,
                                float *d_rot_event, float *d_rot_crystal, void *stream);

/* Parameters of kernel SimulateCrystal (IAC/Simulator.cpp:742-777). */
typedef struct {
    int32_t subsampling;        /* SuSa: (2 SuSa + 1)^2 sub-pixels          */
    double u_step[3];           /* sub-pixel step along the fast axis       */
    double v_step[3];           /* sub-pixel step along the slow axis       */
    double wavelength;
    int32_t intensity_squared;  /* 0: add |Psi| per sub-pixel as the reference
                                   kernel does (IAC/kernel.cl:844); 1: |Psi|^2 */
    int32_t accurate_sincos;    /* 0: explicit 2*pi reduction + SFU sin/cos;
                                   1: sincosf                                */
} iac_sim_params;

/* Kernel SimulateCrystal per mode, summed over modes as SimulatePart does
 * (IAC/Simulator.cpp:779-866), for nframes frames: d_intensity is
 * float[nframes][npix].  Asynchronous. */
iac_status iac_simulate_intensity(iac_ctx *ctx, const float *d_pixel_map, uint64_t npix,
                                  const float *d_emitters, const uint32_t *d_em_count,
                                  uint32_t natoms, uint32_t nmodes, uint32_t nframes,
                                  const iac_sim_params *params, float *d_intensity, void *stream);

/* Post-processing of SimulatePart (IAC/Simulator.cpp:870-894). */
typedef struct {
    double expected_photons;  /* AveragePhotonesPerEmitterOnDetector * FlYield * #atoms */
    int32_t poisson;          /* PoissonSample                                     */
    float adu_noise;          /* ADUNoise (uniform +-level), 0 = none              */
    float value_per_photon;   /* ValuePerPhoton                                    */
} iac_photon_params;

/* Rescale each frame to the expected photon number, draw Poisson counts
 * (inversion below a mean of 25, clipped Box-Muller above, as
 * ArrayOperators::ScalarPoissonSampling), add noise, scale by the value per
 * photon; in place.  Random streams are indexed by first_frame + frame and
 * pixel.  Asynchronous. */
iac_status iac_simulate_photons(iac_ctx *ctx, float *d_intensity, uint64_t npix, uint32_t nframes,
                                uint64_t first_frame, const iac_photon_params *params,
                                uint64_t seed, void *stream);

/* Detector::CreateSparseHitList(Threshold, Step) on the device
 * (IAC/Detector.cpp:926-977) after the pixel mask (IAC/RunIAC.cpp:534):
 * frames float[nframes][npix] -> photon lists float4 (k, value) in pixel order
 * with nframes+1 offsets, ready for iac_sparse_ac_batch.  d_mask may be NULL.
 * If h_total is given the call synchronises, stores the photon count and
 * fails when it exceeds `capacity`.  Entries beyond the capacity are never
 * written and the offsets are clamped to it (counted for iac_ctx_check). */
iac_status iac_sparsify_frames(iac_ctx *ctx, const float *d_intensity, const int *d_mask,
                               const float *d_kmap, uint64_t npix, uint32_t nframes,
                               float threshold, float step, int photonize, float *d_photons,
                               uint64_t capacity, uint64_t *d_frame_offsets, uint64_t *h_total,
                               void *stream);

/* ---------------------------------------------------------------------- */
/* averaged intensity and per-event statistics                               */
/* ---------------------------------------------------------------------- */

/* Detector::LoadAndAverageIntensity (IAC/Detector.cpp:687-790) for a batch of
 * loaded frames [nframes][npix] (fp32, events in order): masked by d_mask
 * (int per pixel, optional), then either thresholded and added to d_sum
 * (step <= 0) or discretised to photons and counted in d_discr (step > 0);
 * d_sum / d_discr accumulate across batches.  Per frame, d_mean_intensity =
 * sequential FP32 sum / npix (the event's MeanIntensity) and, with step > 0,
 * d_photon_sum = the sum itself (PhotonCount = (int)sum).  Bit-exact with the
 * reference.  Asynchronous. */
iac_status iac_average_frames(iac_ctx *ctx, const float *d_frames, uint64_t npix, uint32_t nframes,
                              const int32_t *d_mask, float threshold, float step, float *d_sum,
                              int64_t *d_discr, float *d_mean_intensity, float *d_photon_sum,
                              void *stream);
/* Intensity = (step > 0 ? (float)d_discr : d_sum) * (1 / nframes_total). */
iac_status iac_average_finish(iac_ctx *ctx, const float *d_sum, const int64_t *d_discr, uint64_t npix,
                              uint32_t nframes_total, float *d_intensity, void *stream);

/* ---------------------------------------------------------------------- */
/* mesh denoiser -- no counterpart in the reference                          */
/* ---------------------------------------------------------------------- */

/* A 3-level 3D U-Net (channels 16/32/64, 3x3x3 convolutions, average
 * pooling, nearest upsampling + skip concatenation, residual 1x1 head) that
 * maps a few-frame pair mesh to an estimate of its many-frame mean.  Volumes
 * are fp32 [nb][D][H][W] on the device, D, H, W multiples of 4.  Forward and
 * backward run on hand-written BF16 implicit-GEMM tensor-core kernels with
 * FP32 accumulation; parameters are fp32 (one flat array, per 3x3x3 layer
 * W[cout][27][cin] then b[cout]; head w[16], b) updated by AdamW. */
typedef struct iac_denoiser iac_denoiser;

typedef struct iac_adamw {
    float lr, beta1, beta2, eps, weight_decay;
} iac_adamw;

/* number of fp32 parameters */
uint64_t iac_denoise_param_count(void);

/* Workspace for up to max_batch volumes of D x H x W.  backend 0 runs the
 * convolutions on tcgen05.mma with TMEM accumulators over padded-row slabs
 * (persistent CTAs), 1 on mma.sync, 2 on tcgen05.mma with one gathered
 * operand tile per tap. */
iac_status iac_denoise_create(iac_ctx *ctx, uint32_t max_batch, uint32_t D, uint32_t H, uint32_t W,
                              int backend, iac_denoiser **out);
void iac_denoise_destroy(iac_denoiser *dn);

/* He-normal weights, zero biases and head (identity network); resets AdamW. */
iac_status iac_denoise_init_params(iac_denoiser *dn, uint64_t seed);
/* host fp32 arrays of iac_denoise_param_count() values; set resets AdamW.
 * Synchronous. */
iac_status iac_denoise_set_params(iac_denoiser *dn, const float *h_params);
iac_status iac_denoise_get_params(iac_denoiser *dn, float *h_params);
iac_status iac_denoise_get_grads(iac_denoiser *dn, float *h_grads);
/* The device gradient vector itself (float[*count], the layout of
 * iac_denoise_get_params), which iac_denoise_backward writes and
 * iac_denoise_adamw_step reads, for data-parallel training on several GPUs:
 * between the two calls every rank sums the vector across ranks in place (an
 * NCCL all-reduce) and scales it by 1 / ranks, so that all replicas take the
 * same optimizer step on the mean gradient.  The pointer stays valid until
 * iac_denoise_destroy.  No counterpart in the reference (its output of record
 * is the plain mesh). */
iac_status iac_denoise_grad_buffer(iac_denoiser *dn, float **d_grads, uint64_t *count);
/* Training state for checkpoint/resume (no counterpart in the reference): the
 * AdamW moments (nparams floats each) and step count; set_state restores the
 * parameters, moments and step together (set_params resets the moments). */
iac_status iac_denoise_get_state(iac_denoiser *dn, float *h_m, float *h_v, uint64_t *h_step);
iac_status iac_denoise_set_state(iac_denoiser *dn, const float *h_params, const float *h_m, const float *h_v,
                                 uint64_t step);

/* d_out = network(d_in).  Asynchronous on `stream`. */
iac_status iac_denoise_forward(iac_denoiser *dn, const float *d_in, uint32_t nb, uint32_t D, uint32_t H,
                               uint32_t W, float *d_out, void *stream);

/* Forward, loss = mean(weight * (out - target)^2) (weight may be null), and
 * the parameter gradients (read with iac_denoise_get_grads).  d_out may be
 * null.  When h_loss is given the call synchronizes `stream` and stores the
 * loss there. */
iac_status iac_denoise_backward(iac_denoiser *dn, const float *d_in, const float *d_target,
                                const float *d_weight, uint32_t nb, uint32_t D, uint32_t H, uint32_t W,
                                float *d_out, double *h_loss, void *stream);

/* One AdamW step on the gradients of the last backward.  Asynchronous. */
iac_status iac_denoise_adamw_step(iac_denoiser *dn, const iac_adamw *opt, void *stream);

/* One 3x3x3 convolution layer (stride 1, zero padding 1) on bf16 NDHWC
 * tensors: y = [relu](conv(concat(up0 ? upsample2(src0) : src0, src1)) + bias).
 * src0 (c0 channels, may be absent with c0 = 0) is at half resolution when
 * up0; src1 (c1 channels) and y (cout) are nb x D x H x W.  d_wtile holds the
 * weights W[co][tap][ci] as bf16 tiles [tap][ci/8][co][8] (tap = 9 (dz+1) +
 * 3 (dy+1) + dx+1).  The (cin, cout) pairs of the network are supported.
 * Asynchronous. */
iac_status iac_denoise_conv3x3(iac_ctx *ctx, int backend, const uint16_t *d_src0, uint32_t c0, int up0,
                               const uint16_t *d_src1, uint32_t c1, const uint16_t *d_wtile,
                               const float *d_bias, uint32_t cout, int relu, uint32_t nb, uint32_t D,
                               uint32_t H, uint32_t W, uint16_t *d_y, void *stream);

/* Weight gradient of that layer: d_dw[co][tap][ci] += sum_v grad[v][co] X[v + off(tap)][ci]
 * and d_db[co] += sum_v grad[v][co] (fp32, accumulated; d_db may be null).
 * slabs = 3 runs it on tcgen05 with the three dz planes of a tile stacked
 * into one MMA operand (16/32 input channels: the input slabs along M; 48 in,
 * 16 out: the gradient slabs along N; other shapes as 2), 2 on tcgen05 with
 * one dz per CTA (TMEM accumulators, TMA-fed stages; plain inputs only, else
 * as 1), 1 on mma.sync staging each input row once per tile and dz, 0 on
 * mma.sync with one gathered tile per tap.  Asynchronous. */
iac_status iac_denoise_wgrad3x3(iac_ctx *ctx, int slabs, const uint16_t *d_src0, uint32_t c0, int up0,
                                const uint16_t *d_src1, uint32_t c1, const uint16_t *d_grad,
                                uint32_t cout, uint32_t nb, uint32_t D, uint32_t H, uint32_t W,
                                float *d_dw, float *d_db, void *stream);

/* nsteps training steps replayed from one CUDA graph: per step the patches
 * of plan d_plans[step] ([nsteps][nb][5] int32, as iac_denoise_crop_patches)
 * are cut from the nmeshes E^3 bf16 input and target meshes, the loss and
 * gradients computed and AdamW applied with learning rate d_lrs[step]
 * (opt->lr is ignored).  d_losses (optional, double[nsteps]) receives each
 * step's sum of squared errors.  The graph is captured on the first call and
 * reused while the pointers, sizes and hyper-parameters stay the same.
 * Asynchronous. */
iac_status iac_denoise_train_steps(iac_denoiser *dn, const uint16_t *d_in_meshes,
                                   const uint16_t *d_tgt_meshes, uint32_t nmeshes, uint32_t E,
                                   const int32_t *d_plans, const float *d_lrs, uint32_t nsteps,
                                   uint32_t nb, uint32_t P, const iac_adamw *opt, double *d_losses,
                                   void *stream);

/* Network input from a folded S^3 uint64 mesh: its leading E^3 corner times
 * `scale`, as fp32 (d_f32) and/or bf16 bits (d_bf16).  Asynchronous. */
iac_status iac_denoise_mesh_input(iac_ctx *ctx, const uint64_t *d_full, uint32_t S, uint32_t E,
                                  double scale, float *d_f32, uint16_t *d_bf16, void *stream);

/* Training patches: plan (int32 x 5 per patch: mesh index, z0, y0, x0,
 * transform 0..47 = axis permutation + 6 x reflection bits) cuts P^3 fp32
 * patches from nmeshes E^3 bf16 meshes.  Plan entries reaching outside the
 * meshes give zeros and count as out-of-mesh (iac_ctx_check).  Asynchronous. */
iac_status iac_denoise_crop_patches(iac_ctx *ctx, const uint16_t *d_meshes, uint32_t nmeshes, uint32_t E,
                                    const int32_t *d_plan, uint32_t nb, uint32_t P, float *d_out,
                                    void *stream);

/* ---------------------------------------------------------------------- */
/* micro-benchmarks (roofline denominators)                                 */
/* ---------------------------------------------------------------------- */

/* Scattered 64-bit (or 32-bit) atomic adds into a buffer of `words` words:
 * `updates` adds at pseudo-random addresses.  Used to measure the L2 atomic
 * rate the pair kernels are bound by.  Asynchronous. */
iac_status iac_bench_scatter_add(iac_ctx *ctx, void *d_buffer, uint64_t words, int word_bits,
                                 uint64_t updates, uint32_t seed, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* IAC_B200_H */
