// Internal types shared by the host code and the kernels of libvirs_b200.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "virs.h"

namespace virs {

// ---- errors ----------------------------------------------------------------

void set_error(const std::string &msg);
virs_status fail(virs_status st, const std::string &msg);
virs_status cuda_fail(cudaError_t e, const char *what);

#define VIRS_CUDA(call)                                          \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return ::virs::cuda_fail(e_, #call); \
    } while (0)

#define VIRS_TRY(call)                       \
    do {                                     \
        virs_status s_ = (call);             \
        if (s_ != VIRS_OK) return s_;        \
    } while (0)

// ---- filter states ----------------------------------------------------------
//
// The 2(S+1) filter states of each boundary slot (step_common.cuh) come in
// groups of four, one 16-byte vector per group; group g of every slot is
// one array of vectors, so a warp's consecutive slots read consecutive
// vectors and a slot's states take one vector load per group.  Entry e of
// slot s sits at float index state_index(e, s, nb).
__host__ __device__ inline uint64_t state_index(uint32_t e, uint64_t s, uint64_t nb)
{
    return ((uint64_t)(e >> 2) * nb + s) * 4u + (e & 3u);
}
inline uint32_t state_groups(uint32_t nsec) { return (2u * (nsec + 1u) + 3u) / 4u; }

// ---- device buffer -----------------------------------------------------------

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    virs_status alloc(size_t n, const char *what);   // zero-filled
    template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

// ---- cell codes (one byte per voxel, padded layout) -------------------------
//
// The step kernel reads one byte per voxel instead of seven flags: for air
// and boundary voxels the low six bits say which face neighbours are walls
// (their value is replaced by the centre value, the mirror rule of
// simulator_gpu.cu:70-81) and bit 7 marks a boundary voxel.
constexpr uint8_t CODE_NONE = 0xFF;   // border / padding: never written
constexpr uint8_t CODE_WALL = 0xFE;   // flag 1: p+ = 0
constexpr uint8_t CODE_HARD = 0xFD;   // flag 3: p+ = hard source value
constexpr uint8_t CODE_BND = 0x80;    // flag 2 (with the wall mask in bits 0-5)
// wall-mask bits, in the reference's summation order
constexpr uint8_t W_XP = 1, W_XM = 2, W_YP = 4, W_YM = 8, W_ZP = 16, W_ZM = 32;

constexpr int SEG = 128;              // voxels per boundary-prefix segment

// ---- kernel argument blocks -------------------------------------------------

struct StepArgs {
    float4 *side;           // per boundary slot {free, p, p^{n-1}, 0}, kept by the boundary pass for the adjoint
    const uint32_t *stop;   // nonzero *stop: the RMS stop rule has fired, the step does nothing (nullptr: off)
    const uint64_t *tzmask; // TMA stencil, per tile: bit j = the codes of stage j are all zero (nullptr: none)
    const void *p;          // p^n (storage type)
    void *q;                // in p^{n-1}, out p^{n+1}
    const uint8_t *code;
    const uint8_t *normals; // air-neighbour mask (rigid-wall update)
    const uint32_t *bpos;   // [nb] padded device index of each boundary slot
    const uint8_t *bcode;   // [nb] cell code of each slot's voxel (read in slot order, not gathered)
    const uint8_t *bnrm;    // [nb] air-neighbour mask of each slot's voxel (rigid-wall update)
    const uint8_t *bmat;
    const float *bw;
    float *state;           // X_q[n-1], X_q[n-2] of the cascade's input and section outputs (state_index)
    float *state_out;       // where the pass writes the states after the step (nullptr: in place, `state`)
    const float *coef;      // [M][S][5]
    const float *hard;      // per-step hard source values (scaled)
    const uint32_t *ctr;    // device step counter
    uint64_t nb;
    uint32_t nhard;
    uint32_t nsec;
    uint32_t nx, ny, nz, px;
    int zc;                 // planes per block
    int zb, ze;             // the stencil updates planes [zb, ze): 1 and nz - 1 for a whole step
    int form;               // VIRS_BOUNDARY_*
    float c2dt2, inv_h2;
    float l2;               // (c dt / h)^2 of the rigid-wall update
    int rigid;              // boundary voxels: rigid-wall update instead of the mirrored leapfrog
    int sr;                 // 16-bit storage: stochastic rounding of the stores (step_common.cuh)
    uint64_t sr_base;       // its key offset: a slab's first padded voxel in the whole grid (0 otherwise)
    double K, mix_y, mix_d, gain;
};

struct PostArgs {
    void *q;                // p^{n+1}
    const uint64_t *src;    // device indices
    const float *sig;       // [nsrc][siglen] (scaled)
    const uint64_t *rcv;    // device indices
    float *ir;              // [nrcv][cap]
    uint32_t *ctr;
    uint32_t nsrc, nrcv;
    uint64_t siglen, cap;
    float inv_scale;
    const uint32_t *hpos;   // device positions of the hard-source voxels
    uint32_t nhpos;
    uint32_t nhard;         // per-step hard-source values (scaled) in `hard`
    const float *hard;
    uint32_t *stop;         // the RMS stop rule on the device (nullptr: off): {stopped, stop step, filter state}
    int sr;                 // as StepArgs::sr / sr_base
    uint64_t sr_base;
};

// one member of a batched run (device-resident descriptor)
struct alignas(64) BatchMember {
    CUtensorMap mapP[2];    // halo box over field[0] / field[1]
    CUtensorMap mapQ[2];    // tile box over field[0] / field[1]
    CUtensorMap mapC;       // cell codes
    StepArgs step[2];       // per parity: p = field[parity], q = field[parity ^ 1]
    PostArgs post[2];
    const uint32_t *bidx;
    uint64_t first_tile;    // index of this member's first tile in the batch
    uint64_t first_bnd;     // index of this member's first boundary voxel
    uint32_t gx, gy, gz;    // tile grid
};
cudaError_t launch_step_tma_batch(int storage, int tile_rows, int depth, const BatchMember *mem, uint32_t nmem,
                                  uint64_t ntiles, int parity, bool persistent, int *err, cudaStream_t s, bool sr);
cudaError_t launch_boundary_batch(int storage, const BatchMember *mem, uint32_t nmem, uint64_t nbnd, int parity,
                                  uint32_t max_sections, cudaStream_t s);
cudaError_t launch_post_batch(int storage, const BatchMember *mem, uint32_t nmem, int parity, cudaStream_t s);

// kernel launchers (kernels_step.cu)
cudaError_t launch_step(int storage, int tile_rows, const StepArgs &a, cudaStream_t s);
cudaError_t launch_post(int storage, const PostArgs &a, cudaStream_t s);
// modes of the boundary pass (kernels_step.cu)
enum { BND_UPDATE = 0, BND_KEEP = 1, BND_RECORD = 2 };
cudaError_t launch_boundary(int storage, const StepArgs &a, int mode, cudaStream_t s);
int default_planes(uint32_t nz);

// TMA-staged step (kernels_step_tma.cu)
struct TmaMaps {
    const CUtensorMap *p;   // p^n with halo box
    const CUtensorMap *q;   // p^{n-1}, tile box
    const CUtensorMap *c;   // cell codes, tile box
};
cudaError_t launch_step_tma(int storage, int tile_rows, int depth, const StepArgs &a, const TmaMaps &m, int *err,
                            cudaStream_t s);
int tma_box_width(int storage);   // x extent of the halo box (elements)
int tma_pad(int storage);         // x halo on each side (elements)
int tma_tile_x();                 // x extent of a tile
// two steps in one pass (kernels_step_tma.cu): p^n (a.p, maps m.p) and
// p^{n-1} (a.q, maps m.q) in, p^{n+1} to zout and p^{n+2} to wout; tiles of
// tile_rows (16 or 32) rows, a.zc planes (0: all); then, after the first
// boundary pass and post kernel, launch_boundary_fix (kernels_step.cu) runs
// the second boundary pass (a.p = p^{n+1}, a.q = p^{n+2}) together with the
// recomputation of the p^{n+2} of the voxels in list from p^{n+1} and p^n
cudaError_t launch_pair_tma(int storage, int tile_rows, const StepArgs &a, const TmaMaps &m, void *zout, void *wout,
                            int *err, cudaStream_t s);
cudaError_t launch_boundary_fix(int storage, const StepArgs &a, const void *pn, const uint32_t *list, uint32_t nlist,
                                cudaStream_t s);
int pair_tile_x(int storage);   // inner tile width of the two-step kernel
int pair_code_box();            // width of its code box (bytes)
// the voxels whose p^{n+2} the two-step kernel leaves provisional
// (kernels_classify.cu): marks (zeroed by the caller) and per-segment counts
// of 1024 voxels, then, with the counts scanned, their ascending positions
// per tile of the two-step kernel (inner width ix, vector width v), the
// stages whose codes are all zero (kernels_classify.cu)
cudaError_t launch_pair_zero_masks(const uint8_t *segnz, uint32_t px, uint32_t ny, uint32_t nz, uint32_t spr,
                                   uint32_t rows, uint32_t zc, uint32_t ix, uint32_t v, uint32_t gx, uint32_t gy,
                                   uint32_t gz, uint64_t *mask, cudaStream_t s);
size_t mark_segments(uint64_t nvox);
cudaError_t launch_pair_marks(const uint8_t *code, uint32_t px, uint32_t ny, uint32_t nz, const uint32_t *bpos,
                              uint64_t nb, const uint32_t *hpos, uint32_t nh, const uint64_t *src, uint32_t nsrc,
                              uint8_t *mark, uint32_t *cnt, cudaStream_t s);
cudaError_t launch_mark_list(const uint8_t *mark, uint64_t nvox, const uint32_t *off, uint32_t *list, cudaStream_t s);
cudaError_t launch_wait_probe(int *err, uint32_t limit, cudaStream_t s);

// classification launchers (kernels_classify.cu)
struct ClassifyArgs {
    const uint8_t *flags_in;   // padded
    const uint8_t *wall_mat;   // padded
    uint8_t *flags_out;        // padded
    uint8_t *bmat_full;        // padded scratch
    uint16_t *bd2_full;        // padded scratch
    uint32_t *k1, *k2;         // padded scratch
    uint32_t nx, ny, nz, px;
    int W;
};
cudaError_t launch_sponge(const ClassifyArgs &a, cudaStream_t s);

struct CodesArgs {
    const uint8_t *flags;      // padded, classified
    uint8_t *code;             // padded
    uint8_t *normals;          // padded
    uint32_t *segcnt;          // [nseg]
    uint8_t *segnz;            // [nseg] 1 if the segment holds a non-zero code
    uint32_t nx, ny, nz, px, spr;
};
cudaError_t launch_codes(const CodesArgs &a, cudaStream_t s);
// exclusive scan of n u32 values in place; tmp needs scan_tmp_words(n) words
size_t scan_tmp_words(size_t n);
cudaError_t launch_scan(uint32_t *data, size_t n, uint32_t *tmp, uint32_t *total, cudaStream_t s);

struct CompactArgs {
    const uint8_t *flags;      // padded, classified
    const uint32_t *bseg;
    const uint8_t *bmat_full;
    const uint16_t *bd2_full;
    const float *wtab;         // sponge weight per d2
    uint32_t *bidx;
    uint32_t *bpos;            // padded device index of each slot's voxel
    const uint8_t *code;       // padded cell codes and air-neighbour masks
    const uint8_t *normals;
    uint8_t *bcode, *bnrm;     // ... copied per slot
    uint8_t *bmat;
    float *bw;
    uint32_t nx, ny, nz, px, spr;
};
cudaError_t launch_compact(const CompactArgs &a, cudaStream_t s);
// per tile of a rows x zc tiling of the TMA stencil: bit j set when the codes
// of the plane in stage j are all zero (kernels_classify.cu)
// (planes [zb, ze) in chunks of zc: 1 and nz - 1 for a whole step)
cudaError_t launch_tile_zero_masks(const uint8_t *segnz, uint32_t ny, uint32_t nz, uint32_t spr, uint32_t rows,
                                   uint32_t zc, uint32_t gx, uint32_t gy, uint32_t gz, uint32_t zb, uint32_t ze,
                                   uint64_t *mask, cudaStream_t s);
cudaError_t launch_hard_list(const uint8_t *code, uint64_t n, uint32_t *count, uint32_t *out, uint32_t cap,
                             cudaStream_t s);

// adjoint kernels (kernels_adjoint.cu)
cudaError_t launch_adj_inject(float *T, const uint8_t *code, const uint64_t *rcv, uint32_t nrcv, const float *dl,
                              uint64_t dl_stride, uint64_t n, const uint64_t *src, uint32_t nsrc, float *gsig,
                              uint64_t gs_stride, cudaStream_t s);
cudaError_t launch_adj_boundary(float *T, const uint32_t *bidx, const uint8_t *bmat, const float *bw, const float *coef,
                                const float4 *rec, const float *fst, float *ast, float *dbar, float *cq, double *grad,
                                uint64_t nb, uint32_t nx, uint32_t ny, uint32_t px, uint32_t nsec, uint32_t nmat,
                                int form, double K, double mix_y, double mix_d, double gain, cudaStream_t s);
cudaError_t launch_adj_fix(float *Tn, float *Tb, const uint32_t *bidx, const float4 *rec, const float *dbar,
                           const float *cq, uint64_t nb, uint32_t nx, uint32_t ny, uint32_t px, cudaStream_t s);
cudaError_t launch_set_u32(uint32_t *p, uint32_t v, cudaStream_t s);
cudaError_t launch_zero_at(float *f, const uint32_t *pos, uint32_t n, cudaStream_t s);

// mesh voxelisation (kernels_voxelize.cu)
size_t voxelize_tri_bytes();
cudaError_t launch_voxelize(const float *verts, const uint32_t *tris, const int32_t *tri_mat, uint64_t ntri,
                            const uint8_t *roles, uint32_t nroles, float h, const float bmin[3], uint32_t nx,
                            uint32_t ny, uint32_t nz, uint32_t zw, uint32_t nzl, uint32_t px, void *tri_buf,
                            uint32_t *last_any, uint32_t *last_wall, uint8_t *flags, uint8_t *wall_mat,
                            uint32_t *max_mat, cudaStream_t s);

// IR post-processing (kernels_ir.cu)
cudaError_t launch_ir_sos(const float *in, uint64_t in_stride, uint64_t len, const double *sos, int ns, float *out,
                          uint64_t out_stride, uint32_t channels, cudaStream_t s);
cudaError_t launch_ir_sinc(const float *in, uint64_t in_stride, uint64_t len, double fs_in, double rate, int half,
                           double beta, double cutoff, float *out, uint64_t out_len, uint32_t *peak, uint32_t channels,
                           cudaStream_t s);
cudaError_t launch_ir_resample(const float *in, uint64_t in_stride, uint64_t len, double sim_rate, float rate,
                               float *out, uint64_t out_len, int normalize, uint32_t channels, cudaStream_t s);

// misc kernels (kernels_misc.cu)
cudaError_t launch_energy(int storage, const void *p, const void *q, const uint8_t *code, uint32_t nx, uint32_t ny,
                          uint32_t nz, uint32_t px, double lambda2, double inv_scale2, double *partial,
                          int nblocks, cudaStream_t s);
cudaError_t launch_sphere(int storage, void *p, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px, uint64_t cx,
                          uint64_t cy, uint64_t cz, uint64_t r, float value, int init, cudaStream_t s);
cudaError_t launch_pack(int storage, const void *field, float *out, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t px,
                        float inv_scale, cudaStream_t s);
cudaError_t launch_unpack(int storage, const float *in, void *field, uint32_t nx, uint32_t ny, uint32_t nz,
                          uint32_t px, float scale, cudaStream_t s);

// what virs_energy_noalloc needs from a handle (capi.cpp)
struct EnergyInputs {
    const void *p, *q;
    const uint8_t *code;
    uint32_t nx, ny, nz, px;
    int storage, device;
    double lambda2, scale2;
    cudaStream_t stream;
    cudaEvent_t done; // the handle's completion event, recorded after the launches
};
virs_status energy_inputs(virs_sim *sim, void *stream, EnergyInputs *out);

// ---- host-side geometry (voxelize.cpp, design.cpp) ---------------------------

struct Mesh {
    std::vector<float> verts;          // [n][3]
    std::vector<uint32_t> tris;        // [t][3]
    std::vector<int32_t> tri_mat;      // [t]
};

virs_status load_obj(const char *path, Mesh &out);
void mesh_bbox(const Mesh &m, float nudge, float bmin[3], float bmax[3]);
void grid_dims(const float bmin[3], const float bmax[3], float h, uint64_t dims[3]);


void rbj_highpass(float fs, float cutoff, float q, float gain, float out5[5]);
void rbj_lowpass(float fs, float cutoff, float q, float gain, float out5[5]);
float sponge_weight(int W, int d2);

} // namespace virs
