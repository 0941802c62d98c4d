/*
 * iac_oracle.h -- CPU restatement of IncohAutoCorrelate's pair-correlation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 * The product (libiac_b200.so) never links, calls or falls back to it.
 *
 * Every function restates one piece of the reference, cited as path:line of
 * the FabianTr/IncohAutoCorrelate tree (IncohAutoCorrelate/ is abbreviated IAC/).
 * Arithmetic follows the reference's own operation order and types; the file is
 * compiled with -ffp-contract=off so no multiply-add is fused, and sqrtf is the
 * correctly rounded IEEE square root.  Parity is pinned by tests that compare
 * this restatement with the reference's kernel.cl compiled for the CPU
 * (oracle/_ref) and by the committed golden fixtures under tests/golden/.
 */
#ifndef IAC_ORACLE_H
#define IAC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ACMesh::MeshShape, IAC/ACMesh.h:21-29 */
typedef struct {
    uint32_t k_a, k_b, k_c;
    uint32_t size_ab, size_c;
    uint32_t center[3];
    float dq_per_voxel;
    uint32_t voxel_per_dq;
    float max_q;
} iaco_mesh_shape;

/* AC1D::Shape (IAC/AC1D.h) */
typedef struct {
    uint32_t size;
    float max_q;
    float dq_per_step;
} iaco_ac1d_shape;

/* ---- geometry / mesh sizing ------------------------------------------ */
void iaco_calc_kmap(const float *pixel_map, uint64_t npix, float *kmap, float max_q[3]);
void iaco_generate_pixel_map(int size_a, int size_b, float pixel_size, const float center[3],
                             const float vec_a[3], const float vec_b[3], float *pixel_map);
int iaco_big_mesh_shape(const float max_q[3], int edge_size, float q_zoom, iaco_mesh_shape *s);
int iaco_small_cq_mesh_shape(const float max_q[3], int perp_size, float q_zoom, iaco_mesh_shape *s);
void iaco_ac1d_shape_init(const float max_q[3], uint32_t array_size, float q_zoom, iaco_ac1d_shape *s);

/* ---- photonisation / sparse list ------------------------------------- */
void iaco_discretize_to_photons(float *a, uint64_t n, float threshold, float step);
void iaco_average_frames(const float *frames, uint64_t npix, uint32_t nframes, const int32_t *mask,
                         float threshold, float step, float *sum, int64_t *discr, float *mean_intensity,
                         float *photon_sum);
void iaco_average_finish(const float *sum, const int64_t *discr, uint64_t npix, uint32_t nframes_total,
                         float *intensity);
uint64_t iaco_sparse_hitlist(const float *intensity, const float *kmap, uint64_t npix,
                             float threshold, float step, int photonize, float *out4);

/* ---- (a) sparse photon pairs -> uint64 3D mesh ----------------------- */
/* Device route of one frame: Autocor_sparseHL into a half mesh. */
uint64_t iaco_sparse_ac_halfmesh(const float *hl4, uint32_t n, const double params[9],
                                 const float rot9[9], uint64_t *half);
/* Host fold of the half mesh into the full mesh (FloatToInt of half/Mult). */
void iaco_fold_halfmesh(const uint64_t *half, uint32_t S, double multiplicator, float step,
                        float offset, uint64_t *full);
/* CPU route of one frame: ACMesh::Atomic_Add_q_Entry for i<=j, +q and -q. */
uint64_t iaco_sparse_ac_cpu_route(const float *hl4, uint32_t n, const float rot9[9],
                                  const iaco_mesh_shape *s, int interp1, int interp2,
                                  int double_map, float step, float offset, uint64_t *full);
/* Detector::AutoCorrelateSparseList: route choice + route.  Returns 0 (CPU)
 * or 1 (device route).  half_scratch must hold S*S*((S+1)/2) words. */
int iaco_autocorrelate_sparse_list(const float *hl4, uint32_t n, uint64_t det_pixels,
                                   const float rot9[9], const iaco_mesh_shape *s,
                                   int interp1, int interp2, int double_map, float step,
                                   float offset, int cpu_gpu, uint64_t *half_scratch,
                                   uint64_t *full, uint64_t *oob);
/* Many frames through the device route, each folded on its own (reference
 * semantics of RunIAC's per-frame loop with CpuGpu = 1). */
uint64_t iaco_sparse_ac_batch(const float *hl4, const uint64_t *frame_offsets, uint32_t nframes,
                              const float *rot9, const iaco_mesh_shape *s, int interp1,
                              int interp2, int double_map, float step, float offset,
                              int cpu_gpu, uint64_t det_pixels, uint64_t *full);

/* ---- (b) dense mean-intensity C(q) ----------------------------------- */
double iaco_cq_small_multiplicator(const float *intensity, uint64_t npix);
uint64_t iaco_cq_small(const float *intensity, const float *kmap, uint64_t npix,
                       const iaco_mesh_shape *s, int interp, double multiplicator,
                       uint64_t row_begin, uint64_t row_end, uint64_t *mesh);
void iaco_cq_merge_weights(const float *rot9_all, const float *mean_intensity, uint32_t nframes,
                           const double *small_cq, uint64_t small_n, float *rw10,
                           double *multiplicator);
uint64_t iaco_cq_merge(const double *small_cq, const float *rw10, uint32_t nframes,
                       const iaco_mesh_shape *small_shape, int interp, double multiplicator,
                       uint64_t voxel_begin, uint64_t voxel_end, uint64_t *big);

/* ---- (c) AC1D -------------------------------------------------------- */
double iaco_ac1d_cq_multiplicator(const float *intensity, uint64_t npix);
/* AutoCorr_CQ_AV summed over its 10000 sub-histograms (integer totals). */
uint64_t iaco_ac1d_cq(const float *intensity, const float *kmap, uint64_t npix,
                      const iaco_ac1d_shape *s, int interp, double multiplicator,
                      uint64_t row_begin, uint64_t row_end, uint64_t *hist);
/* AutoCorr_sparseHL_AAV of one frame, integer totals folded modulo VecSize. */
uint32_t iaco_ac1d_vecsize(float max_q, float dqdx);
void iaco_ac1d_sparse_frame(const float *hl4, uint32_t n, float max_q, float dqdx, int interp,
                            double multiplicator, uint64_t *hist_vecsize);
/* CPU route of Calculate_AC_UW_Mapped (k >= j, factor 2), double accumulation. */
void iaco_ac1d_sparse_frame_cpu_route(const float *hl4, uint32_t n, float max_q, float dqdx,
                                      int interp, double *ac);

/* Both routes of Calculate_AC_UW_Mapped over frames (route -1: the
 * reference's per-frame choice, 0: CPU loop, 1: device kernel). */
void iaco_ac1d_uw_frames(const float *hl4, const uint64_t *frame_offsets, uint32_t nframes,
                         uint64_t det_pixels, float max_q, float dqdx, uint32_t size, int interp,
                         int route, double *ac);

/* ---- (d) simulator --------------------------------------------------- */
void iaco_simulate_crystal(const float *pixel_map, uint64_t npix, const float *em4, uint32_t nem,
                           const double params[10], int intensity_mode, float *out);
void iaco_simulate_crystal_f64(const float *pixel_map, uint64_t npix, const float *em4,
                               uint32_t nem, const double params[10], int intensity_mode,
                               double *out);
void iaco_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double iaco_uniform_double(uint64_t seed, uint64_t stream, uint64_t idx, uint32_t draw);
uint32_t iaco_poisson(double mean, uint64_t seed, uint64_t stream, uint64_t idx);
void iaco_poisson_array(const float *mean, uint64_t n, uint64_t seed, uint64_t stream,
                        float *out);
void iaco_crystal_lattice(const double lattice_vec[9], const uint32_t cells[3],
                          const double *unit_cell, uint32_t n_uc, double *atoms);
void iaco_rotation_axis_angle(double alpha, const double axis[3], float rot9[9]);
void iaco_invert3(const float m[9], float inv[9]);

/* ---- final merge ----------------------------------------------------- */
void iaco_merge_ac_and_cq(const uint64_t *ac, const double *cq, uint64_t n, float step,
                          float offset, double *out);

#ifdef __cplusplus
}
#endif
#endif
