// The C ABI of include/virs.h: one handle per simulation, all device memory
// owned by the handle, every failure returned as a status with a message.
//
// Flow (the reference's, simulator.cpp:262-1025):
//   virs_create -> virs_load_obj / virs_set_mesh / virs_set_grid
//   -> virs_classify (GPU: sponge layer, normals, codes, boundary list)
//   -> virs_set_filters / virs_set_sources / virs_set_receivers
//   -> virs_start_simulation -> virs_run (graph) or virs_step (per step)
//   -> virs_get_ir -> virs_destroy
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <new>
#include <string>
#include <deque>
#include <vector>

#include <cudaTypedefs.h>

#include "internal.hpp"

#define VIRS_EXPORT extern "C" __attribute__((visibility("default")))

namespace virs {

namespace {
thread_local std::string g_err;
}

void set_error(const std::string &msg) { g_err = msg; }

virs_status fail(virs_status st, const std::string &msg)
{
    g_err = msg;
    return st;
}

virs_status cuda_fail(cudaError_t e, const char *what)
{
    g_err = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return VIRS_E_OOM;
    return VIRS_E_CUDA;
}

virs_status DevBuf::alloc(size_t n, const char *what)
{
    release();
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return fail(VIRS_E_OOM, std::string("cudaMalloc of ") + std::to_string(n) + " bytes for " + what + " failed: " +
                                    cudaGetErrorString(e));
    }
    bytes = n;
    e = cudaMemsetAsync(ptr, 0, n, cudaStreamPerThread);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemset");
    return VIRS_OK;
}

// Every copy and memset of the library runs on the handle's own stream, a
// non-blocking stream, and is complete when the call returns: nothing goes
// to the legacy default stream, which would have to wait for (and would
// break) a graph capture in progress on another handle's stream in another
// host thread.
cudaError_t copy_on(cudaStream_t st, void *dst, const void *src, size_t n, cudaMemcpyKind k)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, n, k, st);
    return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}

cudaError_t copy2d_on(cudaStream_t st, void *dst, size_t dpitch, const void *src, size_t spitch, size_t w, size_t h,
                      cudaMemcpyKind k)
{
    cudaError_t e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, w, h, k, st);
    return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}

cudaError_t zero_on(cudaStream_t st, void *p, size_t n)
{
    cudaError_t e = cudaMemsetAsync(p, 0, n, st);
    return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}

} // namespace virs

using namespace virs;

namespace virs {
namespace {
// a number no other handle of this process carries
uint64_t next_handle_id()
{
    static std::atomic<uint64_t> n{0};
    return ++n;
}
} // namespace
} // namespace virs

// the step graph of a virs_slab_run over the same slabs (kept by the first
// slab): valid while every slab is the same handle, unchanged (gen), and
// at the buffer parity it was captured for
struct SlabGraph {
    std::vector<const virs_sim *> mem;
    std::vector<uint64_t> id, gen;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    ~SlabGraph()
    {
        for (cudaGraphExec_t g : exec)
            if (g) cudaGraphExecDestroy(g);
    }
};

struct virs_sim {
    const uint64_t id = virs::next_handle_id();
    virs_params prm{};
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::unique_ptr<SlabGraph> slab_graph;

    // geometry
    bool has_grid = false, classified = false;
    uint32_t nx = 0, ny = 0, nz = 0, px = 0, spr = 0;
    size_t nvox = 0;      // padded voxels
    size_t nref = 0;      // nx*ny*nz
    float h = 0.f;
    float bmin[3] = {0, 0, 0};
    std::vector<uint8_t> roles;
    uint8_t max_wall_mat = 0;

    DevBuf flags_raw, wall_mat, flags, code, normals, bseg;
    DevBuf segnz;                  // [nseg] 1 if a 128-voxel row segment holds a non-zero code
    DevBuf field[2];
    int cur = 0;

    // z-slab of a larger grid (virs_set_grid_slab): flags_raw / wall_mat
    // hold ext_nz planes, classified together; the grid kept (nz planes,
    // the owned planes and a ghost plane each side) starts slab_drop planes
    // into them.  For a whole grid ext_nz == nz and slab_drop == 0.
    bool slab = false;
    cudaStream_t xstream = nullptr;    // virs_slab_run: the ghost-plane pulls, beside the interior stencil
    cudaEvent_t xdone = nullptr;       // ... and their completion
    int rounding = VIRS_ROUND_NEAREST; // of the 16-bit stores (virs_set_rounding)
    uint32_t ext_nz = 0, slab_drop = 0;
    uint64_t slab_lo = 0, slab_hi = 0, global_nz = 0; // owned global planes and the global grid's planes

    // boundary
    uint64_t nb = 0;
    DevBuf bidx, bpos, bcode, bnrm, bmat, bw, state;
    DevBuf hpos;                   // hard-source voxel positions
    uint32_t nhpos = 0;

    // filters
    uint32_t nmat = 0, nsec = 0;
    DevBuf coef;
    bool filters_set = false;

    // sources / receivers
    DevBuf hard;
    uint32_t nhard = 0;
    std::vector<float> hard_host;
    DevBuf src, sig;
    uint32_t nsrc = 0;
    uint64_t siglen = 0;
    std::vector<uint64_t> src_ref;
    std::vector<float> sig_host;   // unscaled [nsrc][siglen]
    float sig_peak = 0.f;
    DevBuf rcv;
    uint32_t nrcv = 0;
    std::vector<uint64_t> rcv_ref;
    DevBuf ir;
    uint64_t ircap = 0;
    DevBuf ctr;
    uint64_t steps_done = 0;

    // constants
    float dt = 0, c2dt2 = 0, inv_h2 = 0, K = 0, l2 = 0;
    double fs = 0;
    float scale = 1.f, inv_scale = 1.f;

    // kernel variant: depth 0 = register-streaming kernel, 1..3 = TMA
    // kernel with that many planes in flight
    int tile_rows = 8, zc = 0, depth = 2;
    CUtensorMap tmP[2], tmQ[2], tmC;
    DevBuf side;                   // {free, p, p^{n-1}} per boundary slot (TMA kernel -> boundary pass)
    int maps_rows = 0;             // tile rows the maps were built for (0 = none)
    // per stencil tile, the stages whose codes are all zero (not copied);
    // built for zm_rows x zm_zc tiles (0 = none)
    DevBuf zmask;
    int zm_rows = 0, zm_zc = 0;
    // the same for the slab-interior launch of virs_slab_run (planes 2 .. nz-3)
    DevBuf zmask_in;
    int zmi_rows = 0, zmi_zc = 0;
    DevBuf err;                    // device error flag of bounded waits

    // two steps per pass (virs_set_time_blocking).  spare[k] is the partner
    // of field[k] in a four-buffer rotation (four steps go field -> spare ->
    // field); pmP / pmQ are the maps of field[0], field[1], spare[0],
    // spare[1] (index 0..3) for pm_rows-row tiles, pmC the wider code box;
    // plist holds the voxels whose second step is provisional (pl_ok: built
    // for the current codes and sources)
    int pair_steps = 1, pair_rows = 14, pair_zc = 0;
    DevBuf spare[2];
    CUtensorMap pmP[4], pmQ[4], pmC;
    int pm_rows = 0;
    DevBuf plist;
    uint32_t nplist = 0;
    bool pl_ok = false;
    DevBuf pzmask;                 // zero-code masks of the two-step tiles (pm_rows x pzm_zc; -1 = none)
    int pzm_zc = -1;
    bool pair_nomem = false;       // the spare buffers did not fit: single steps

    // CUDA graphs for GRAPH_STEPS steps, one per parity of `cur`
    static constexpr int GRAPH_STEPS = 32;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graph_dirty = true;
    uint64_t gen = 0;              // bumped on every change of buffers or parameters

    // timing
    bool timing = false;
    double t_ms = 0, t_bms = 0;
    uint64_t t_steps = 0, t_launch = 0;

    // virs_step's RMS rule (simulator_gpu.cu:303-330)
    std::vector<float> out0;
    float rms_state = 0.f;
    // the same rule on the device for virs_run / virs_run_host
    // (virs_set_stop_rule): {stopped, stop step, filter state}
    DevBuf stopbuf;
    bool stop_rule = false, stopped = false;
    uint64_t stop_step = 0;

    DevBuf energy_partial;

    // adjoint: checkpoints of a forward run and the reverse-pass buffers
    struct {
        uint64_t steps = 0, nck = 0, gen = 0;
        uint32_t every = 0;
        bool ready = false;
        DevBuf ckp, ckq, cks, segrec, segst, buf[2], ast, dbar, cq, grad, dl, gsig;
        CUtensorMap mapP[2], mapQ[2];
    } adj;
    bool fields_valid = true;      // false after virs_adjoint until the next start
    bool slab_open = false;        // virs_slab_step_begin ran, virs_slab_step_end not yet

    ~virs_sim()
    {
        drop_graphs();
        slab_graph.reset();
        if (done) cudaEventDestroy(done);
        if (xdone) cudaEventDestroy(xdone);
        if (xstream) cudaStreamDestroy(xstream);
        if (stream) cudaStreamDestroy(stream);
    }

    void drop_graphs()
    {
        for (auto &g : graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        graph_dirty = true;
        ++gen;
    }

    size_t storage_bytes() const { return prm.storage == VIRS_STORAGE_F32 ? 4 : 2; }
};

namespace {

bool finite_pos(float v) { return std::isfinite(v) && v > 0.f; }

virs_status use_device(const virs_sim *s)
{
    VIRS_CUDA(cudaSetDevice(s->prm.device));
    return VIRS_OK;
}

// step constants, simulator_gpu.cu:195-198 and :147, simulator.cpp:940-952
void compute_constants(virs_sim *s)
{
    const float c = s->prm.sound_speed, h = s->h;
    s->dt = s->prm.courant * h / (c * std::sqrt(3.f));
    s->c2dt2 = c * c * s->dt * s->dt;
    s->inv_h2 = 1.f / (h * h);
    s->K = s->prm.boundary_k != 0.f ? s->prm.boundary_k : (c * s->dt) / h * 0.95f;
    // the rigid-wall update's (c dt / dx)^2 (simulator_gpu.cu:165)
    const float cdh = c * s->dt / h;
    s->l2 = cdh * cdh;
    const double dtd = (double)s->prm.courant * (double)h / ((double)c * std::sqrt(3.0));
    s->fs = 1.f / dtd;
}

virs_status upload_hard(virs_sim *s)
{
    std::vector<float> v(s->hard_host.size());
    for (size_t i = 0; i < v.size(); ++i) v[i] = s->hard_host[i] * s->scale;
    VIRS_TRY(s->hard.alloc(v.size() * sizeof(float), "hard source schedule"));
    if (!v.empty()) VIRS_CUDA(copy_on(s->stream, s->hard.ptr, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice));
    s->nhard = (uint32_t)v.size();
    s->graph_dirty = true;
    ++s->gen;
    return VIRS_OK;
}

// reference default filter: RBJ high-pass 440 Hz, Q 0.1 at fs = 1/dt
// (simulator.cpp:955-967)
virs_status default_filters(virs_sim *s)
{
    float k[5];
    rbj_highpass((float)s->fs, 440.f, 0.1f, 1.f, k);
    s->nmat = 1;
    s->nsec = 1;
    VIRS_TRY(s->coef.alloc(5 * sizeof(float), "filter coefficients"));
    VIRS_CUDA(copy_on(s->stream, s->coef.ptr, k, sizeof(k), cudaMemcpyHostToDevice));
    s->filters_set = true;
    return VIRS_OK;
}

// the filter states: state_groups vectors of four floats per slot (internal.hpp)
size_t state_bytes(const virs_sim *s) { return std::max<uint64_t>(s->nb, 1) * state_groups(s->nsec) * 4 * sizeof(float); }

virs_status alloc_states(virs_sim *s)
{
    VIRS_TRY(s->state.alloc(state_bytes(s), "filter states"));
    s->graph_dirty = true;
    ++s->gen;
    return VIRS_OK;
}

uint64_t to_dev(const virs_sim *s, uint64_t ref)
{
    const uint64_t x = ref % s->nx, y = (ref / s->nx) % s->ny, z = ref / ((uint64_t)s->nx * s->ny);
    return (z * s->ny + y) * s->px + x;
}

bool interior(const virs_sim *s, uint64_t ref)
{
    const uint64_t x = ref % s->nx, y = (ref / s->nx) % s->ny, z = ref / ((uint64_t)s->nx * s->ny);
    return x > 0 && y > 0 && z > 0 && x + 1 < s->nx && y + 1 < s->ny && z + 1 < s->nz;
}

// pitched copies between the reference layout (rows of nx) and the device
// layout (rows of px)
virs_status h2d_rows(void *dst, const void *src, size_t elem, const virs_sim *s, size_t planes = 0)
{
    VIRS_CUDA(copy2d_on(s->stream, dst, (size_t)s->px * elem, src, (size_t)s->nx * elem, (size_t)s->nx * elem,
                           (size_t)s->ny * (planes ? planes : s->nz), cudaMemcpyHostToDevice));
    return VIRS_OK;
}

virs_status d2h_rows(void *dst, const void *src, size_t elem, const virs_sim *s)
{
    VIRS_CUDA(copy2d_on(s->stream, dst, (size_t)s->nx * elem, src, (size_t)s->px * elem, (size_t)s->nx * elem,
                           (size_t)s->ny * s->nz, cudaMemcpyDeviceToHost));
    return VIRS_OK;
}

virs_status wait_done(const virs_sim *s)
{
    VIRS_CUDA(cudaEventSynchronize(s->done));
    return VIRS_OK;
}

// allocate the grid-sized buffers and upload flags / wall materials.  For a
// slab (keep > 0) the nz planes uploaded are classified together and the
// grid kept is `keep` planes from `drop` on.
virs_status install_grid(virs_sim *s, uint64_t nx, uint64_t ny, uint64_t nz, float h, const uint8_t *flags,
                         const uint8_t *wmat, uint64_t keep = 0, uint64_t drop = 0)
{
    if (nx < 3 || ny < 3 || nz < 3) return fail(VIRS_E_ARG, "grid must be at least 3 voxels along each axis");
    if (keep && (keep < 3 || drop + keep > nz)) return fail(VIRS_E_ARG, "slab planes outside the uploaded range");
    if (nx > (1u << 30) || ny > (1u << 30) || nz > (1u << 30) || ((nx + 31) / 32 * 32) * ny * nz >= (1ull << 32))
        return fail(VIRS_E_ARG, "grid too large: voxel positions are 32-bit (nx rounded up to 32, times ny*nz, < 2^32)");
    if (!finite_pos(h)) return fail(VIRS_E_ARG, "cell size must be finite and positive");
    const size_t n = nx * ny * nz;
    uint8_t mx = 0;
    if (flags)
        for (size_t i = 0; i < n; ++i)
            if (flags[i] > 3) return fail(VIRS_E_ARG, "flags must be 0..3 (flag " + std::to_string(flags[i]) + " at " + std::to_string(i) + ")");
    if (wmat)
        for (size_t i = 0; i < n; ++i) mx = std::max(mx, wmat[i]);
    s->drop_graphs();
    s->has_grid = s->classified = false;
    s->slab = keep != 0;
    s->ext_nz = (uint32_t)nz;
    s->slab_drop = (uint32_t)drop;
    if (keep) nz = keep;
    s->nx = (uint32_t)nx;
    s->ny = (uint32_t)ny;
    s->nz = (uint32_t)nz;
    s->px = (uint32_t)((nx + 31) / 32 * 32);
    // segments per row, padded to a multiple of 4 so that rows of the prefix
    // array are 16-byte aligned for the TMA
    s->spr = ((s->px + SEG - 1) / SEG + 3) / 4 * 4;
    s->nvox = (size_t)s->px * ny * nz;
    s->nref = (size_t)nx * ny * nz;
    s->h = h;
    s->max_wall_mat = mx;
    compute_constants(s);
    // release the old grid first so that peak memory stays at one grid
    for (DevBuf *b : {&s->flags_raw, &s->wall_mat, &s->flags, &s->code, &s->normals, &s->bseg, &s->segnz, &s->field[0],
                      &s->field[1], &s->bidx, &s->bpos, &s->bcode, &s->bnrm, &s->bmat, &s->bw, &s->state, &s->side, &s->hpos,
                      &s->spare[0], &s->spare[1], &s->plist, &s->pzmask})
        b->release();
    const size_t ext = (size_t)s->px * ny * s->ext_nz;
    VIRS_TRY(s->flags_raw.alloc(ext, "flags"));
    VIRS_TRY(s->wall_mat.alloc(ext, "wall materials"));
    if (flags) VIRS_TRY(h2d_rows(s->flags_raw.ptr, flags, 1, s, s->ext_nz));
    if (wmat) VIRS_TRY(h2d_rows(s->wall_mat.ptr, wmat, 1, s, s->ext_nz));
    VIRS_TRY(s->flags.alloc(s->nvox, "classified flags"));
    VIRS_TRY(s->field[0].alloc(s->nvox * s->storage_bytes(), "pressure field"));
    VIRS_TRY(s->field[1].alloc(s->nvox * s->storage_bytes(), "pressure field"));
    s->cur = 0;
    s->nb = 0;
    s->steps_done = 0;
    s->maps_rows = 0;
    s->zm_rows = s->zm_zc = 0;
    s->zmi_rows = s->zmi_zc = 0;
    s->pm_rows = 0;
    s->pl_ok = false;
    s->pair_nomem = false;
    // sources and receivers refer to voxel indices of the previous grid
    s->nsrc = s->nrcv = 0;
    s->src_ref.clear();
    s->rcv_ref.clear();
    s->has_grid = true;
    return VIRS_OK;
}

// mesh -> grid: bounding box and sizing on the host, the triangle sweep on
// the GPU (kernels_voxelize.cu) straight into the padded flag arrays
// the interior planes 1..nz-2 split into `parts` contiguous ranges whose
// sizes differ by at most one; range `part` (virs_b200/slabs.py:split_planes)
void split_planes(uint64_t nz, uint32_t part, uint32_t parts, uint64_t *z_lo, uint64_t *z_hi)
{
    const uint64_t inner = nz - 2, base = inner / parts, extra = inner % parts;
    *z_lo = 1 + part * base + std::min<uint64_t>(part, extra);
    *z_hi = *z_lo + base + (part < extra ? 1 : 0);
}

// planes of flags a slab needs on each side of its own grid for the sponge
// classification of its planes: the ghost plane is classified too, and a
// voxel's class depends on the walls within W planes
uint64_t slab_halo(const virs_sim *s) { return (uint64_t)s->prm.sponge_width + 1; }

// parts == 0: the whole grid; otherwise slab `part` of `parts`, whose
// uploaded planes (its own, the ghost planes and the classification halo)
// alone are voxelised, with the whole grid's origin and sizes
virs_status install_mesh(virs_sim *s, const Mesh &m, uint32_t part = 0, uint32_t parts = 0)
{
    float bmin[3], bmax[3];
    mesh_bbox(m, s->prm.bbox_nudge, bmin, bmax);
    const float h = s->prm.cell_size > 0.f ? s->prm.cell_size : 343.f / (22050.f * 2.f * 2.f);
    uint64_t d[3];
    grid_dims(bmin, bmax, h, d);
    if (d[0] < 3 || d[1] < 3 || d[2] < 3) return fail(VIRS_E_ARG, "mesh bounding box gives a grid below 3 voxels per axis");
    if (!parts && d[0] * d[1] * d[2] >= (1ull << 32)) return fail(VIRS_E_ARG, "mesh gives a grid of 2^32 voxels or more");
    uint64_t z_lo = 0, z_hi = 0, z_first = 0, nz_ext = d[2];
    if (parts) {
        if (part >= parts || d[2] - 2 < parts)
            return fail(VIRS_E_ARG, "slab " + std::to_string(part) + " of " + std::to_string(parts) + ": the grid has " +
                                        std::to_string(d[2] - 2) + " interior planes");
        if (s->prm.storage != VIRS_STORAGE_F32 && !(s->prm.storage_scale > 0.f))
            return fail(VIRS_E_ARG, "slabs with 16-bit storage need an explicit storage_scale, the same on every slab");
        split_planes(d[2], part, parts, &z_lo, &z_hi);
        const uint64_t H = slab_halo(s);
        z_first = z_lo - 1 >= H ? z_lo - 1 - H : 0;
        nz_ext = std::min<uint64_t>(d[2], z_hi + 1 + H) - z_first;
    }
    const uint64_t ntri = m.tri_mat.size();
    if (ntri >= 0xffffffffull) return fail(VIRS_E_ARG, "too many triangles");
    for (uint32_t v : m.tris)
        if ((uint64_t)v * 3 + 2 >= m.verts.size()) return fail(VIRS_E_ARG, "triangle vertex index out of range");
    VIRS_TRY(use_device(s));
    if (parts) {
        VIRS_TRY(install_grid(s, d[0], d[1], nz_ext, h, nullptr, nullptr, z_hi - z_lo + 2, z_lo - 1 - z_first));
        s->slab_lo = z_lo;
        s->slab_hi = z_hi;
        s->global_nz = d[2];
    } else {
        VIRS_TRY(install_grid(s, d[0], d[1], d[2], h, nullptr, nullptr));
    }
    std::memcpy(s->bmin, bmin, sizeof(bmin));
    if (ntri) {
        const size_t nvx = (size_t)s->px * s->ny * s->ext_nz; // the uploaded planes
        DevBuf dv, dt, dm, dr, tri, la, lw, mx;
        VIRS_TRY(dv.alloc(m.verts.size() * sizeof(float), "mesh vertices"));
        VIRS_TRY(dt.alloc(m.tris.size() * sizeof(uint32_t), "mesh triangles"));
        VIRS_TRY(dm.alloc(ntri * sizeof(int32_t), "triangle materials"));
        VIRS_TRY(dr.alloc(std::max<size_t>(s->roles.size(), 1), "material roles"));
        VIRS_TRY(tri.alloc(ntri * voxelize_tri_bytes(), "triangle table"));
        VIRS_TRY(la.alloc(nvx * sizeof(uint32_t), "voxelisation marks"));
        VIRS_TRY(lw.alloc(nvx * sizeof(uint32_t), "voxelisation marks"));
        VIRS_TRY(mx.alloc(sizeof(uint32_t), "wall material maximum"));
        VIRS_CUDA(copy_on(s->stream, dv.ptr, m.verts.data(), dv.bytes, cudaMemcpyHostToDevice));
        VIRS_CUDA(copy_on(s->stream, dt.ptr, m.tris.data(), dt.bytes, cudaMemcpyHostToDevice));
        VIRS_CUDA(copy_on(s->stream, dm.ptr, m.tri_mat.data(), dm.bytes, cudaMemcpyHostToDevice));
        if (!s->roles.empty()) VIRS_CUDA(copy_on(s->stream, dr.ptr, s->roles.data(), s->roles.size(), cudaMemcpyHostToDevice));
        VIRS_CUDA(launch_voxelize(dv.as<float>(), dt.as<uint32_t>(), dm.as<int32_t>(), ntri, dr.as<uint8_t>(),
                                  (uint32_t)s->roles.size(), h, bmin, s->nx, s->ny, (uint32_t)d[2], (uint32_t)z_first,
                                  s->ext_nz, s->px, tri.ptr,
                                  la.as<uint32_t>(), lw.as<uint32_t>(), s->flags_raw.as<uint8_t>(),
                                  s->wall_mat.as<uint8_t>(), mx.as<uint32_t>(), s->stream));
        uint32_t mxh = 0;
        VIRS_CUDA(cudaMemcpyAsync(&mxh, mx.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
        VIRS_CUDA(cudaStreamSynchronize(s->stream));
        s->max_wall_mat = (uint8_t)mxh;
    }
    return VIRS_OK;
}

virs_status ensure_ir(virs_sim *s, uint64_t need)
{
    if (need <= s->ircap) return VIRS_OK;
    uint64_t cap = std::max<uint64_t>(need, s->ircap ? s->ircap * 2 : 1024);
    DevBuf nb;
    VIRS_TRY(nb.alloc(std::max<uint32_t>(s->nrcv, 1) * cap * sizeof(float), "receiver samples"));
    if (s->ircap && s->nrcv)
        VIRS_CUDA(copy2d_on(s->stream, nb.ptr, cap * sizeof(float), s->ir.ptr, s->ircap * sizeof(float),
                               s->ircap * sizeof(float), s->nrcv, cudaMemcpyDeviceToDevice));
    std::swap(s->ir.ptr, nb.ptr);
    std::swap(s->ir.bytes, nb.bytes);
    s->ircap = cap;
    s->graph_dirty = true;
    ++s->gen;
    return VIRS_OK;
}

// looked up once, in a static initialiser (thread-safe: handles may be
// created and retiled from several host threads)
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return nullptr;
    }();
    return fn;
}

virs_status encode_dims(CUtensorMap *m, CUtensorMapDataType dt, size_t elem, void *base, uint64_t d0, uint64_t d1,
                        uint64_t d2, uint32_t bx, uint32_t by)
{
    auto fn = encode_fn();
    if (!fn) return fail(VIRS_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {(cuuint64_t)d0 * elem, (cuuint64_t)d0 * d1 * elem};
    const cuuint32_t box[3] = {bx, by, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(m, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VIRS_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return VIRS_OK;
}

// a [nz][ny][px] array of the grid
virs_status encode(CUtensorMap *m, CUtensorMapDataType dt, size_t elem, void *base, const virs_sim *s, uint32_t bx,
                   uint32_t by)
{
    return encode_dims(m, dt, elem, base, s->px, s->ny, s->nz, bx, by);
}

// tensor maps of the two field buffers (halo box and tile box) and of the
// cell codes, for the current tile height
virs_status build_maps(virs_sim *s)
{
    const int rows = s->tile_rows;
    const CUtensorMapDataType dt = s->prm.storage == VIRS_STORAGE_F32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : s->prm.storage == VIRS_STORAGE_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                                        : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const size_t el = s->storage_bytes();
    for (int b = 0; b < 2; ++b) {
        VIRS_TRY(encode(&s->tmP[b], dt, el, s->field[b].ptr, s, (uint32_t)tma_box_width(s->prm.storage), rows + 2));
        VIRS_TRY(encode(&s->tmQ[b], dt, el, s->field[b].ptr, s, (uint32_t)tma_tile_x(), rows));
    }
    VIRS_TRY(encode(&s->tmC, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, s->code.ptr, s, (uint32_t)tma_tile_x(), rows));
    if (!s->err.ptr) VIRS_TRY(s->err.alloc(sizeof(int), "error flag"));
    s->maps_rows = rows;
    return VIRS_OK;
}

// read and clear the device error flag of the bounded waits
virs_status check_err(virs_sim *s)
{
    if (!s->err.ptr) return VIRS_OK;
    int e = 0;
    VIRS_CUDA(copy_on(s->stream, &e, s->err.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        VIRS_CUDA(zero_on(s->stream, s->err.ptr, sizeof(int)));
        return fail(VIRS_E_TIMEOUT, "a stencil block gave up waiting for its staged planes (bounded wait expired)");
    }
    return VIRS_OK;
}

// the SMs of a device (looked up once per device)
int sm_count(int dev)
{
    static std::atomic<int> cache[64];
    if (dev < 0 || dev >= 64) return 148;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            n = 148;
        }
        cache[dev].store(n, std::memory_order_relaxed);
        v = n;
    }
    return v;
}

// planes per block of a single simulation's stencil when none is set: the
// batch default (32), or fewer, down to 4, on grids whose 32-plane tiling
// would give the device fewer than about eight blocks per SM (a 128^3 grid
// has 16 tiles of 128 x 8 voxels per plane: 48 blocks with 32 planes, 384
// with 4)
int eff_planes(const virs_sim *s)
{
    if (s->zc > 0) return s->zc;
    const uint64_t tiles = (uint64_t)((s->px + 127) / 128) * ((s->ny + s->tile_rows - 1) / s->tile_rows);
    const uint64_t want = 8ull * (uint64_t)sm_count(s->prm.device);
    const uint64_t zc = (uint64_t)(s->nz > 2 ? s->nz - 2 : 1) * tiles / want;
    return (int)std::min<uint64_t>(std::max<uint64_t>(zc, 4), (uint64_t)default_planes(s->nz));
}

// per tile of a rows x zc tiling of the TMA stencil, the stages whose codes
// are all zero (kernels_classify.cu::k_tile_zero_mask)
// (planes [zb, ze); 0, 0 = the whole step's planes 1 .. nz-2)
virs_status build_zero_masks(const virs_sim *s, int rows, int zc, DevBuf &mask, uint32_t zb = 0, uint32_t ze = 0)
{
    if (zb == 0 && ze == 0) {
        zb = 1;
        ze = s->nz - 1;
    }
    const uint32_t gx = (s->px + (uint32_t)tma_tile_x() - 1) / (uint32_t)tma_tile_x();
    const uint32_t gy = (s->ny + (uint32_t)rows - 1) / (uint32_t)rows;
    const uint32_t gz = (ze - zb + (uint32_t)zc - 1) / (uint32_t)zc;
    VIRS_TRY(mask.alloc(std::max<size_t>((size_t)gx * gy * gz, 1) * 8, "zero-code masks"));
    VIRS_CUDA(launch_tile_zero_masks(s->segnz.as<uint8_t>(), s->ny, s->nz, s->spr, (uint32_t)rows, (uint32_t)zc, gx,
                                     gy, gz, zb, ze, mask.as<uint64_t>(), s->stream));
    VIRS_CUDA(cudaStreamSynchronize(s->stream));
    return VIRS_OK;
}

// The first and last tile columns hold the grid's border (code CODE_NONE),
// so only grids at least three tiles wide have planes of a tile with all
// codes zero; for the others the masks would cost their tests for nothing.
bool zero_masks_useful(const virs_sim *s) { return s->px > 2u * (uint32_t)tma_tile_x(); }

bool zero_masks_ready(const virs_sim *s)
{
    return s->depth > 0 && zero_masks_useful(s) && s->zm_rows == s->tile_rows && s->zm_zc == eff_planes(s);
}

virs_status ready_to_run(virs_sim *s)
{
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid: call virs_load_obj, virs_set_mesh or virs_set_grid");
    if (!s->classified) return fail(VIRS_E_STATE, "grid not classified: call virs_classify");
    if (!s->filters_set) VIRS_TRY(default_filters(s));
    if (s->nb && s->max_wall_mat >= s->nmat)
        return fail(VIRS_E_ARG, "wall material " + std::to_string(s->max_wall_mat) + " has no filter (" +
                                    std::to_string(s->nmat) + " materials set)");
    if (!s->state.ptr) VIRS_TRY(alloc_states(s));
    if (!s->ctr.ptr) VIRS_TRY(s->ctr.alloc(sizeof(uint32_t), "step counter"));
    if (s->depth > 0 && s->maps_rows != s->tile_rows) VIRS_TRY(build_maps(s));
    if (s->depth > 0 && zero_masks_useful(s) && !zero_masks_ready(s)) {
        s->zm_rows = s->zm_zc = 0;
        VIRS_TRY(build_zero_masks(s, s->tile_rows, eff_planes(s), s->zmask));
        s->zm_rows = s->tile_rows;
        s->zm_zc = eff_planes(s);
        s->drop_graphs();
    }
    return VIRS_OK;
}

// stochastic rounding of the 16-bit stores, and its key offset: a slab's
// voxels take the keys of the same voxels of the whole grid
bool sr_on(const virs_sim *s) { return s->rounding == VIRS_ROUND_STOCHASTIC && s->prm.storage != VIRS_STORAGE_F32; }
uint64_t sr_base(const virs_sim *s) { return s->slab ? (s->slab_lo - 1) * (uint64_t)s->ny * s->px : 0; }

StepArgs step_args(const virs_sim *s, int parity)
{
    StepArgs a{};
    a.sr = sr_on(s) ? 1 : 0;
    a.sr_base = sr_base(s);
    a.side = s->side.as<float4>();
    a.p = s->field[parity].ptr;
    a.q = s->field[parity ^ 1].ptr;
    a.code = s->code.as<uint8_t>();
    a.normals = s->normals.as<uint8_t>();
    a.bpos = s->bpos.as<uint32_t>();
    a.l2 = s->l2;
    a.rigid = s->prm.rigid_walls ? 1 : 0;
    if (s->stop_rule) a.stop = s->stopbuf.as<uint32_t>();
    a.bmat = s->bmat.as<uint8_t>();
    a.bcode = s->bcode.as<uint8_t>();
    a.bnrm = s->bnrm.as<uint8_t>();
    a.bw = s->bw.as<float>();
    a.state = s->state.as<float>();
    a.state_out = nullptr;
    a.coef = s->coef.as<float>();
    a.hard = s->hard.as<float>();
    a.ctr = s->ctr.as<uint32_t>();
    a.nb = s->nb;
    a.nhard = s->nhard;
    a.nsec = s->nsec;
    a.nx = s->nx;
    a.ny = s->ny;
    a.nz = s->nz;
    a.px = s->px;
    a.zc = eff_planes(s);
    a.zb = 1;
    a.ze = (int)s->nz - 1;
    a.c2dt2 = s->c2dt2;
    a.inv_h2 = s->inv_h2;
    a.K = (double)s->K;
    a.mix_y = s->prm.mix_filtered;
    a.mix_d = s->prm.mix_direct;
    a.gain = (double)s->prm.boundary_gain;
    a.form = s->prm.boundary_form;
    if (zero_masks_ready(s)) a.tzmask = s->zmask.as<uint64_t>();
    return a;
}

PostArgs post_args(const virs_sim *s, int parity)
{
    PostArgs a{};
    a.sr = sr_on(s) ? 1 : 0;
    a.sr_base = sr_base(s);
    a.q = s->field[parity ^ 1].ptr;
    if (s->stop_rule) a.stop = s->stopbuf.as<uint32_t>();
    a.src = s->src.as<uint64_t>();
    a.sig = s->sig.as<float>();
    a.rcv = s->rcv.as<uint64_t>();
    a.ir = s->ir.as<float>();
    a.ctr = s->ctr.as<uint32_t>();
    a.nsrc = s->nsrc;
    a.nrcv = s->nrcv;
    a.siglen = s->siglen;
    a.cap = s->ircap;
    a.inv_scale = s->inv_scale;
    a.hpos = s->hpos.as<uint32_t>();
    a.nhpos = s->nhpos;
    a.hard = s->hard.as<float>();
    a.nhard = s->nhard;
    return a;
}

cudaError_t launch_stencil(const virs_sim *s, int parity, cudaStream_t st)
{
    if (s->depth == 0) return launch_step(s->prm.storage, s->tile_rows, step_args(s, parity), st);
    const TmaMaps m{&s->tmP[parity], &s->tmQ[parity ^ 1], &s->tmC};
    return launch_step_tma(s->prm.storage, s->tile_rows, s->depth, step_args(s, parity), m, s->err.as<int>(), st);
}

// the stencil over planes [zb, ze) only (the all-zero code masks belong to
// the whole-step tiling and are not used)
cudaError_t launch_stencil_range(const virs_sim *s, int parity, cudaStream_t st, int zb, int ze)
{
    StepArgs a = step_args(s, parity);
    a.zb = zb;
    a.ze = ze;
    const bool inner = zb == 2 && ze == (int)s->nz - 2 && s->depth > 0 && s->zmi_rows == s->tile_rows &&
                       s->zmi_zc == eff_planes(s);
    a.tzmask = inner ? s->zmask_in.as<uint64_t>() : nullptr;
    if (s->depth == 0) return launch_step(s->prm.storage, s->tile_rows, a, st);
    const TmaMaps m{&s->tmP[parity], &s->tmQ[parity ^ 1], &s->tmC};
    return launch_step_tma(s->prm.storage, s->tile_rows, s->depth, a, m, s->err.as<int>(), st);
}

cudaError_t enqueue_step(const virs_sim *s, int parity, cudaStream_t st)
{
    cudaError_t e = launch_stencil(s, parity, st);
    if (e != cudaSuccess) return e;
    e = launch_boundary(s->prm.storage, step_args(s, parity), BND_UPDATE, st);
    if (e != cudaSuccess) return e;
    return launch_post(s->prm.storage, post_args(s, parity), st);
}

// ---- two steps per pass -------------------------------------------------------

// buffer k of the four-buffer rotation: field[0], field[1], spare[0], spare[1]
void *buf_ptr(const virs_sim *s, int k) { return k < 2 ? s->field[k].ptr : s->spare[k - 2].ptr; }

bool pair_on(const virs_sim *s)
{
    return s->pair_steps == 2 && !s->pair_nomem && !sr_on(s) && s->depth > 0 && s->nx >= 3 && s->ny >= 3 &&
           s->nz >= 3;
}

// the voxels whose p^{n+2} the two-step kernel leaves provisional, for the
// current codes, boundary list and sources (kernels_classify.cu)
virs_status build_pair_list(virs_sim *s)
{
    cudaStream_t st = s->stream;
    const size_t nseg = mark_segments(s->nvox);
    DevBuf mark, cnt, tmp, total;
    VIRS_TRY(mark.alloc(s->nvox, "provisional-voxel marks"));
    VIRS_TRY(cnt.alloc(nseg * 4, "provisional-voxel counts"));
    VIRS_TRY(tmp.alloc(scan_tmp_words(nseg) * 4, "scan scratch"));
    VIRS_TRY(total.alloc(4, "provisional-voxel total"));
    VIRS_CUDA(cudaMemsetAsync(mark.ptr, 0, s->nvox, st));
    VIRS_CUDA(launch_pair_marks(s->code.as<uint8_t>(), s->px, s->ny, s->nz, s->bpos.as<uint32_t>(), s->nb,
                                s->hpos.as<uint32_t>(), s->nhpos, s->src.as<uint64_t>(), s->nsrc, mark.as<uint8_t>(),
                                cnt.as<uint32_t>(), st));
    VIRS_CUDA(launch_scan(cnt.as<uint32_t>(), nseg, tmp.as<uint32_t>(), total.as<uint32_t>(), st));
    uint32_t n = 0;
    VIRS_CUDA(cudaMemcpyAsync(&n, total.ptr, 4, cudaMemcpyDeviceToHost, st));
    VIRS_CUDA(cudaStreamSynchronize(st));
    VIRS_TRY(s->plist.alloc(std::max<uint32_t>(n, 1) * 4, "provisional-voxel list"));
    if (n) VIRS_CUDA(launch_mark_list(mark.as<uint8_t>(), s->nvox, cnt.as<uint32_t>(), s->plist.as<uint32_t>(), st));
    VIRS_CUDA(cudaStreamSynchronize(st));
    s->nplist = n;
    s->pl_ok = true;
    s->drop_graphs();
    return VIRS_OK;
}

// spare buffers, maps and the provisional-voxel list; a grid whose spare
// buffers do not fit in device memory runs single steps
virs_status ready_pairs(virs_sim *s)
{
    const size_t fb = s->nvox * s->storage_bytes();
    for (int k = 0; k < 2; ++k)
        if (!s->spare[k].ptr && s->spare[k].alloc(fb, "pressure field (rotation)") != VIRS_OK) {
            s->spare[0].release();
            s->spare[1].release();
            (void)cudaGetLastError();
            s->pair_nomem = true;
            s->drop_graphs();
            return VIRS_OK;
        }
    if (s->pm_rows != s->pair_rows) {
        const int rows = s->pair_rows;
        const CUtensorMapDataType dt = s->prm.storage == VIRS_STORAGE_F32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                       : s->prm.storage == VIRS_STORAGE_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                                            : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
        const size_t el = s->storage_bytes();
        for (int b = 0; b < 4; ++b) {
            VIRS_TRY(encode(&s->pmP[b], dt, el, buf_ptr(s, b), s, (uint32_t)tma_box_width(s->prm.storage), rows + 2));
            VIRS_TRY(encode(&s->pmQ[b], dt, el, buf_ptr(s, b), s, (uint32_t)tma_tile_x(), rows));
        }
        VIRS_TRY(encode(&s->pmC, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, s->code.ptr, s, (uint32_t)pair_code_box(), rows));
        if (!s->err.ptr) VIRS_TRY(s->err.alloc(sizeof(int), "error flag"));
        s->pm_rows = rows;
        s->pzm_zc = -1;
        s->drop_graphs();
    }
    if (zero_masks_useful(s) && s->pzm_zc != s->pair_zc) {
        const uint32_t ix = (uint32_t)pair_tile_x(s->prm.storage), v = (uint32_t)(16 / s->storage_bytes());
        const uint32_t rows = (uint32_t)s->pair_rows, zc = s->pair_zc > 0 ? (uint32_t)s->pair_zc : s->nz - 2;
        const uint32_t gx = (s->px + ix - 1) / ix, gy = (s->ny + rows - 3) / (rows - 2);
        const uint32_t gz = (s->nz - 2 + zc - 1) / zc;
        VIRS_TRY(s->pzmask.alloc((size_t)gx * gy * gz * 8, "two-step zero-code masks"));
        VIRS_CUDA(launch_pair_zero_masks(s->segnz.as<uint8_t>(), s->px, s->ny, s->nz, s->spr, rows, zc, ix, v, gx, gy,
                                         gz, s->pzmask.as<uint64_t>(), s->stream));
        VIRS_CUDA(cudaStreamSynchronize(s->stream));
        s->pzm_zc = s->pair_zc;
        s->drop_graphs();
    }
    if (!s->pl_ok) VIRS_TRY(build_pair_list(s));
    return VIRS_OK;
}

// The planes z = 0 and nz-1 keep their values (border codes) and no stencil
// writes them: spare[k] takes those of field[k], its partner in the rotation.
virs_status sync_border_planes(virs_sim *s, cudaStream_t st)
{
    const size_t pb = (size_t)s->px * s->ny * s->storage_bytes(), last = (size_t)(s->nz - 1) * pb;
    for (int k = 0; k < 2; ++k) {
        VIRS_CUDA(cudaMemcpyAsync(s->spare[k].ptr, s->field[k].ptr, pb, cudaMemcpyDeviceToDevice, st));
        VIRS_CUDA(cudaMemcpyAsync(s->spare[k].as<char>() + last, s->field[k].as<char>() + last, pb,
                                  cudaMemcpyDeviceToDevice, st));
    }
    return VIRS_OK;
}

StepArgs step_args_bufs(const virs_sim *s, int p, int q)
{
    StepArgs a = step_args(s, 0);
    a.p = buf_ptr(s, p);
    a.q = buf_ptr(s, q);
    a.tzmask = nullptr;
    return a;
}

PostArgs post_args_buf(const virs_sim *s, int q)
{
    PostArgs a = post_args(s, 0);
    a.q = buf_ptr(s, q);
    return a;
}

// Two steps: p^n in buffer x, p^{n-1} in y; p^{n+1} to z, p^{n+2} to w.
// After k_pair_tma the first step is completed (boundary pass, post kernel);
// then one launch runs the second step's boundary pass and recomputes its
// provisional voxels, and the second post kernel follows.
cudaError_t enqueue_pair(const virs_sim *s, int x, int y, int z, int w, cudaStream_t st, cudaEvent_t *ev = nullptr)
{
    const int sto = s->prm.storage;
    StepArgs a = step_args_bufs(s, x, y);
    a.zc = s->pair_zc;
    if (zero_masks_useful(s) && s->pzm_zc == s->pair_zc) a.tzmask = s->pzmask.as<uint64_t>();
    const TmaMaps m{&s->pmP[x], &s->pmQ[y], &s->pmC};
    if (ev) cudaEventRecord(ev[0], st);
    cudaError_t e = launch_pair_tma(sto, s->pair_rows, a, m, buf_ptr(s, z), buf_ptr(s, w), s->err.as<int>(), st);
    if (ev) cudaEventRecord(ev[1], st);
    if (e == cudaSuccess) e = launch_boundary(sto, step_args_bufs(s, x, z), BND_UPDATE, st);
    if (ev) cudaEventRecord(ev[2], st);
    if (e == cudaSuccess) e = launch_post(sto, post_args_buf(s, z), st);
    if (ev) cudaEventRecord(ev[3], st);
    if (e == cudaSuccess)
        e = launch_boundary_fix(sto, step_args_bufs(s, z, w), buf_ptr(s, x), s->plist.as<uint32_t>(), s->nplist, st);
    if (ev) cudaEventRecord(ev[4], st);
    if (e == cudaSuccess) e = launch_post(sto, post_args_buf(s, w), st);
    return e;
}

// four steps from parity par, field -> spare -> field: the state is back in
// field[par] (p^n) and field[par ^ 1] (p^{n-1}) afterwards
cudaError_t enqueue_quad(const virs_sim *s, int par, cudaStream_t st, cudaEvent_t *ev = nullptr)
{
    cudaError_t e = enqueue_pair(s, par, par ^ 1, 2 + (par ^ 1), 2 + par, st, ev);
    if (e == cudaSuccess) e = enqueue_pair(s, 2 + par, 2 + (par ^ 1), par ^ 1, par, st, ev ? ev + 5 : nullptr);
    return e;
}

// kernels per pair: the two-step kernel, two post kernels, the first
// boundary pass, and the second one together with the fix-up
uint64_t pair_launches(const virs_sim *s) { return 3 + (s->nb ? 1 : 0) + (s->nb || s->nplist ? 1 : 0); }

virs_status build_graphs(virs_sim *s, cudaStream_t st)
{
    s->drop_graphs();
    for (int par = 0; par < 2; ++par) {
        cudaGraph_t g = nullptr;
        VIRS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        if (pair_on(s))
            for (int i = 0; i < virs_sim::GRAPH_STEPS / 4 && e == cudaSuccess; ++i) e = enqueue_quad(s, par, st);
        else
            for (int i = 0; i < virs_sim::GRAPH_STEPS && e == cudaSuccess; ++i) e = enqueue_step(s, par ^ (i & 1), st);
        cudaError_t e2 = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(e, "capturing the step loop");
        }
        if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&s->graph[par], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    }
    s->graph_dirty = false;
    return VIRS_OK;
}

// The stop rule fired after step `ran` of a run whose first 4*quads steps
// went through the four-buffer rotation from parity par: every later kernel
// returned at entry, so the last step's p and p^{n-1} are where that step
// left them.  Put them back into field[cur] and field[cur ^ 1] (cur = par ^
// (ran & 1)), the layout the rest of the library reads.
virs_status settle_pair_stop(virs_sim *s, int par, uint64_t ran, cudaStream_t st)
{
    const size_t fb = s->field[0].bytes;
    auto copy = [&](int k) { return cudaMemcpyAsync(s->field[k].ptr, s->spare[k].ptr, fb, cudaMemcpyDeviceToDevice, st); };
    switch ((ran - 1) % 4) {
    case 0: VIRS_CUDA(copy(par ^ 1)); break;     // p: spare[par^1]; p^{n-1}: field[par]
    case 1:                                       // p: spare[par]; p^{n-1}: spare[par^1]
        VIRS_CUDA(copy(par));
        VIRS_CUDA(copy(par ^ 1));
        break;
    case 2: VIRS_CUDA(copy(par)); break;         // p: field[par^1]; p^{n-1}: spare[par]
    default: break;                              // a whole group: the usual layout
    }
    VIRS_CUDA(cudaStreamSynchronize(st));
    return VIRS_OK;
}

virs_status run_steps(virs_sim *s, uint64_t n, cudaStream_t st)
{
    if (s->stop_rule && s->stopped) return VIRS_OK; // nothing runs after the rule fired, until a new start
    if (!s->fields_valid) return fail(VIRS_E_STATE, "the fields were consumed by virs_adjoint: start the simulation again");
    VIRS_TRY(ready_to_run(s));
    VIRS_TRY(ensure_ir(s, s->steps_done + n));
    // with two steps per pass, whole groups of four steps go through the
    // spare buffers and back; the remaining n % 4 are single steps
    uint64_t quads = 0;
    if (pair_on(s) && n >= 4) {
        VIRS_TRY(ready_pairs(s));
        if (pair_on(s)) {
            quads = n / 4;
            VIRS_TRY(sync_border_planes(s, st));
        }
    }
    const uint64_t n1 = n - 4 * quads; // single steps, after the quads (which keep the parity)
    if (s->timing) {
        cudaError_t err = cudaSuccess;
        if (quads) {
            std::vector<cudaEvent_t> ev(10 * quads);
            for (auto &e : ev) VIRS_CUDA(cudaEventCreate(&e));
            for (uint64_t q = 0; q < quads && err == cudaSuccess; ++q) err = enqueue_quad(s, s->cur, st, &ev[10 * q]);
            if (err == cudaSuccess) err = cudaStreamSynchronize(st);
            double ms = 0, bms = 0;
            for (uint64_t p = 0; p < 2 * quads && err == cudaSuccess; ++p) {
                float t = 0, b1 = 0, b2 = 0;
                err = cudaEventElapsedTime(&t, ev[5 * p], ev[5 * p + 1]);
                if (err == cudaSuccess) err = cudaEventElapsedTime(&b1, ev[5 * p + 1], ev[5 * p + 2]);
                if (err == cudaSuccess) err = cudaEventElapsedTime(&b2, ev[5 * p + 3], ev[5 * p + 4]);
                ms += t;
                bms += (double)b1 + b2;
            }
            for (auto &e : ev) cudaEventDestroy(e);
            if (err != cudaSuccess) return cuda_fail(err, "timed two-step loop");
            s->t_ms += ms;
            s->t_bms += bms;
            s->t_steps += 2 * quads;
            s->t_launch += 2 * quads * pair_launches(s);
        }
        if (n1) {
            std::vector<cudaEvent_t> ev(3 * n1);
            for (auto &e : ev) VIRS_CUDA(cudaEventCreate(&e));
            for (uint64_t i = 0; i < n1 && err == cudaSuccess; ++i) {
                const int par = s->cur ^ (int)(i & 1);
                cudaEventRecord(ev[2 * i], st);
                err = launch_stencil(s, par, st);
                cudaEventRecord(ev[2 * i + 1], st);
                if (err == cudaSuccess) err = launch_boundary(s->prm.storage, step_args(s, par), BND_UPDATE, st);
                cudaEventRecord(ev[2 * n1 + i], st);
                if (err == cudaSuccess) err = launch_post(s->prm.storage, post_args(s, par), st);
            }
            if (err == cudaSuccess) err = cudaStreamSynchronize(st);
            double ms = 0, bms = 0;
            for (uint64_t i = 0; i < n1 && err == cudaSuccess; ++i) {
                float t = 0, tb = 0;
                err = cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
                if (err == cudaSuccess) err = cudaEventElapsedTime(&tb, ev[2 * i + 1], ev[2 * n1 + i]);
                ms += t;
                bms += tb;
            }
            for (auto &e : ev) cudaEventDestroy(e);
            if (err != cudaSuccess) return cuda_fail(err, "timed step loop");
            s->t_ms += ms;
            s->t_bms += bms;
            s->t_steps += n1;
            s->t_launch += (s->nb ? 3 : 2) * n1;
        }
    } else {
        uint64_t i = 0;
        if (quads) {
            constexpr uint64_t GQ = virs_sim::GRAPH_STEPS / 4;
            uint64_t q = 0;
            if (quads >= GQ) {
                if (s->graph_dirty) VIRS_TRY(build_graphs(s, st));
                for (; q + GQ <= quads; q += GQ) VIRS_CUDA(cudaGraphLaunch(s->graph[s->cur], st));
            }
            for (; q < quads; ++q) {
                cudaError_t e = enqueue_quad(s, s->cur, st);
                if (e != cudaSuccess) return cuda_fail(e, "two-step launch");
            }
        } else if (n >= (uint64_t)virs_sim::GRAPH_STEPS) {
            if (s->graph_dirty) VIRS_TRY(build_graphs(s, st));
            for (; i + virs_sim::GRAPH_STEPS <= n; i += virs_sim::GRAPH_STEPS)
                VIRS_CUDA(cudaGraphLaunch(s->graph[s->cur ^ (int)(i & 1)], st));
        }
        for (uint64_t k = 0; k < n1 - i; ++k) {
            cudaError_t e = enqueue_step(s, s->cur ^ (int)((i + k) & 1), st);
            if (e != cudaSuccess) return cuda_fail(e, "step launch");
        }
    }
    const int cur0 = s->cur;
    const uint64_t done0 = s->steps_done;
    s->cur ^= (int)(n & 1);
    s->steps_done += n;
    VIRS_CUDA(cudaEventRecord(s->done, st));
    if (s->stop_rule) {
        // how many of the n steps ran before the rule fired
        uint32_t sb[2] = {0, 0};
        VIRS_CUDA(cudaMemcpyAsync(sb, s->stopbuf.ptr, sizeof(sb), cudaMemcpyDeviceToHost, st));
        VIRS_CUDA(cudaStreamSynchronize(st));
        if (sb[0]) {
            const uint64_t ran = (uint64_t)sb[1] + 1 - done0;
            s->cur = cur0 ^ (int)(ran & 1);
            s->steps_done = (uint64_t)sb[1] + 1;
            s->stopped = true;
            s->stop_step = sb[1];
            if (ran <= 4 * quads) VIRS_TRY(settle_pair_stop(s, cur0, ran, st));
        }
    }
    return VIRS_OK;
}

} // namespace

// ============================================================================
// exported entry points
// ============================================================================

VIRS_EXPORT const char *virs_last_error(void) { return g_err.c_str(); }

VIRS_EXPORT virs_status virs_params_default(virs_params *p)
{
    if (!p) return fail(VIRS_E_ARG, "virs_params_default: null");
    std::memset(p, 0, sizeof(*p));
    p->struct_size = sizeof(virs_params);
    p->device = 0;
    p->sound_speed = 343.f;
    p->courant = 0.5f;
    p->cell_size = 0.f;
    p->bbox_nudge = 0.1f;
    p->sponge_width = 1;
    p->storage = VIRS_STORAGE_F32;
    p->boundary_form = VIRS_BOUNDARY_REFERENCE;
    p->storage_scale = 0.f;
    p->boundary_gain = 0.4f;
    p->boundary_k = 0.f;
    p->mix_filtered = 0.1;
    p->mix_direct = 0.9;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_create(const virs_params *p, virs_sim **out)
{
    if (!out) return fail(VIRS_E_ARG, "virs_create: null output");
    *out = nullptr;
    virs_params prm;
    if (p) {
        if (p->struct_size != sizeof(virs_params))
            return fail(VIRS_E_ARG, "virs_params.struct_size mismatch (header and library disagree)");
        prm = *p;
    } else {
        virs_params_default(&prm);
    }
    if (!finite_pos(prm.sound_speed)) return fail(VIRS_E_ARG, "sound speed must be positive");
    if (!finite_pos(prm.courant) || prm.courant > 1.f)
        return fail(VIRS_E_ARG, "courant must be in (0, 1]: dt = courant*h/(c*sqrt(3)) and 1 is the 3D stability limit");
    if (!(prm.cell_size >= 0.f) || !std::isfinite(prm.cell_size)) return fail(VIRS_E_ARG, "cell size must be >= 0");
    if (prm.sponge_width < 1 || prm.sponge_width > 31) return fail(VIRS_E_ARG, "sponge width must be 1..31");
    if (prm.storage < VIRS_STORAGE_F32 || prm.storage > VIRS_STORAGE_BF16) return fail(VIRS_E_ARG, "unknown storage");
    if (prm.boundary_form != VIRS_BOUNDARY_REFERENCE && prm.boundary_form != VIRS_BOUNDARY_CENTERED)
        return fail(VIRS_E_ARG, "unknown boundary form");
    if (!(prm.storage_scale >= 0.f) || !std::isfinite(prm.storage_scale)) return fail(VIRS_E_ARG, "storage scale must be >= 0");
    if (prm.rigid_walls != 0 && prm.rigid_walls != 1) return fail(VIRS_E_ARG, "rigid_walls must be 0 or 1");
    int ndev = 0;
    VIRS_CUDA(cudaGetDeviceCount(&ndev));
    if (prm.device < 0 || prm.device >= ndev) return fail(VIRS_E_ARG, "no CUDA device " + std::to_string(prm.device));
    std::unique_ptr<virs_sim> s(new (std::nothrow) virs_sim());
    if (!s) return fail(VIRS_E_OOM, "virs_create: host allocation failed");
    s->prm = prm;
    VIRS_TRY(use_device(s.get()));
    // a blocking stream: it orders after the synchronous copies and memsets
    // of the setup calls, which run on the legacy default stream
    VIRS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    VIRS_CUDA(cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming));
    VIRS_CUDA(cudaEventRecord(s->done, s->stream));
    s->roles.assign(2, VIRS_ROLE_IGNORE);
    s->roles[0] = 0;
    s->roles[1] = VIRS_ROLE_SOURCE;
    // simulator_gpu.cu:214-218: 10 for the first 10 steps
    s->hard_host.assign(10, 10.f);
    *out = s.release();
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_destroy(virs_sim *s)
{
    if (!s) return VIRS_OK;
    cudaSetDevice(s->prm.device);
    // the last work queued for the handle, on its own stream or a caller's
    if (s->done) cudaEventSynchronize(s->done);
    cudaStreamSynchronize(s->stream);
    delete s;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_material_roles(virs_sim *s, const uint8_t *roles, size_t n)
{
    if (!s || (!roles && n)) return fail(VIRS_E_ARG, "virs_set_material_roles: null argument");
    for (size_t i = 0; i < n; ++i)
        if (roles[i] >= 64 && roles[i] != VIRS_ROLE_IGNORE && roles[i] != VIRS_ROLE_SOURCE)
            return fail(VIRS_E_ARG, "role must be 0..63, VIRS_ROLE_SOURCE or VIRS_ROLE_IGNORE");
    s->roles.assign(roles, roles + n);
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_load_obj(virs_sim *s, const char *path)
{
    if (!s || !path) return fail(VIRS_E_ARG, "virs_load_obj: null argument");
    VIRS_TRY(use_device(s));
    Mesh m;
    VIRS_TRY(load_obj(path, m));
    return install_mesh(s, m);
}

static virs_status set_mesh(virs_sim *s, const float *verts, size_t nverts, const uint32_t *tris,
                            const int32_t *tri_material, size_t ntris, uint32_t part, uint32_t parts)
{
    if (!s || !verts || !tris || !tri_material || !nverts || !ntris)
        return fail(VIRS_E_ARG, "virs_set_mesh: null or empty argument");
    VIRS_TRY(use_device(s));
    Mesh m;
    m.verts.assign(verts, verts + 3 * nverts);
    m.tris.assign(tris, tris + 3 * ntris);
    m.tri_mat.assign(tri_material, tri_material + ntris);
    for (uint32_t v : m.tris)
        if (v >= nverts) return fail(VIRS_E_ARG, "virs_set_mesh: triangle vertex index out of range");
    for (float v : m.verts)
        if (!std::isfinite(v)) return fail(VIRS_E_ARG, "virs_set_mesh: non-finite vertex coordinate");
    return install_mesh(s, m, part, parts);
}

VIRS_EXPORT virs_status virs_set_mesh(virs_sim *s, const float *verts, size_t nverts, const uint32_t *tris,
                                      const int32_t *tri_material, size_t ntris)
{
    return set_mesh(s, verts, nverts, tris, tri_material, ntris, 0, 0);
}

VIRS_EXPORT virs_status virs_set_mesh_slab(virs_sim *s, const float *verts, size_t nverts, const uint32_t *tris,
                                           const int32_t *tri_material, size_t ntris, uint32_t part, uint32_t parts)
{
    if (!parts) return fail(VIRS_E_ARG, "virs_set_mesh_slab: parts must be at least 1");
    return set_mesh(s, verts, nverts, tris, tri_material, ntris, part, parts);
}

VIRS_EXPORT virs_status virs_load_obj_slab(virs_sim *s, const char *path, uint32_t part, uint32_t parts)
{
    if (!s || !path) return fail(VIRS_E_ARG, "virs_load_obj_slab: null argument");
    if (!parts) return fail(VIRS_E_ARG, "virs_load_obj_slab: parts must be at least 1");
    VIRS_TRY(use_device(s));
    Mesh m;
    VIRS_TRY(load_obj(path, m));
    return install_mesh(s, m, part, parts);
}

VIRS_EXPORT virs_status virs_get_slab_info(const virs_sim *s, uint64_t *z_lo, uint64_t *z_hi, uint64_t *nz)
{
    if (!s || !z_lo || !z_hi || !nz) return fail(VIRS_E_ARG, "virs_get_slab_info: null argument");
    if (!s->slab) return fail(VIRS_E_STATE, "virs_get_slab_info: not a slab");
    *z_lo = s->slab_lo;
    *z_hi = s->slab_hi;
    *nz = s->global_nz;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_grid(virs_sim *s, uint64_t nx, uint64_t ny, uint64_t nz, float h,
                                      const uint8_t *flags, const uint8_t *wmat)
{
    if (!s || !flags) return fail(VIRS_E_ARG, "virs_set_grid: null argument");
    VIRS_TRY(use_device(s));
    VIRS_TRY(install_grid(s, nx, ny, nz, h, flags, wmat));
    s->bmin[0] = s->bmin[1] = s->bmin[2] = 0.f;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_grid_slab(virs_sim *s, uint64_t nx, uint64_t ny, uint64_t nz, float h, uint64_t z_lo,
                                           uint64_t z_hi, const uint8_t *flags, const uint8_t *wmat, uint64_t z_first,
                                           uint64_t nz_ext)
{
    if (!s || !flags) return fail(VIRS_E_ARG, "virs_set_grid_slab: null argument");
    if (nz < 3 || z_lo < 1 || z_hi <= z_lo || z_hi > nz - 1)
        return fail(VIRS_E_ARG, "virs_set_grid_slab: owned planes must satisfy 1 <= z_lo < z_hi <= nz - 1");
    const uint64_t H = slab_halo(s);
    const uint64_t need_lo = z_lo - 1 >= H ? z_lo - 1 - H : 0;
    const uint64_t need_hi = std::min<uint64_t>(nz, z_hi + 1 + H);
    if (z_first > need_lo || z_first + nz_ext < need_hi || z_first + nz_ext > nz)
        return fail(VIRS_E_ARG, "virs_set_grid_slab: flags must cover planes " + std::to_string(need_lo) + ".." +
                                    std::to_string(need_hi - 1) + " (the slab, its ghost planes and sponge width + 1 "
                                    "planes beyond) and stay inside the grid");
    if (s->prm.storage != VIRS_STORAGE_F32 && !(s->prm.storage_scale > 0.f))
        return fail(VIRS_E_ARG, "virs_set_grid_slab: 16-bit storage needs an explicit storage_scale, the same on every slab");
    VIRS_TRY(use_device(s));
    VIRS_TRY(install_grid(s, nx, ny, nz_ext, h, flags, wmat, z_hi - z_lo + 2, z_lo - 1 - z_first));
    s->slab_lo = z_lo;
    s->slab_hi = z_hi;
    s->global_nz = nz;
    s->bmin[0] = s->bmin[1] = s->bmin[2] = 0.f;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_slab_planes(const virs_sim *s, void **first, void **last, void **ghost_lo,
                                         void **ghost_hi, size_t *plane_bytes)
{
    if (!s || !first || !last || !ghost_lo || !ghost_hi || !plane_bytes)
        return fail(VIRS_E_ARG, "virs_slab_planes: null argument");
    if (!s->slab) return fail(VIRS_E_STATE, "virs_slab_planes: not a slab (virs_set_grid_slab)");
    const size_t pb = (size_t)s->px * s->ny * s->storage_bytes();
    char *p = s->field[s->cur].as<char>(); // p^n: the state the next step reads
    *ghost_lo = p;
    *first = p + pb;
    *last = p + (size_t)(s->nz - 2) * pb;
    *ghost_hi = p + (size_t)(s->nz - 1) * pb;
    *plane_bytes = pb;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_grid_info(const virs_sim *s, virs_grid_info *o)
{
    if (!s || !o) return fail(VIRS_E_ARG, "virs_get_grid_info: null argument");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    o->nx = s->nx;
    o->ny = s->ny;
    o->nz = s->nz;
    o->cell_size = s->h;
    std::memcpy(o->bbox_min, s->bmin, sizeof(s->bmin));
    o->dt = s->dt;
    o->sample_rate = s->fs;
    o->boundary_count = s->nb;
    o->steps_done = s->steps_done;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_classify(virs_sim *s)
{
    if (!s) return fail(VIRS_E_ARG, "virs_classify: null");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    s->drop_graphs();
    s->classified = false;
    cudaStream_t st = s->stream;
    const int W = s->prm.sponge_width;
    {
        // the sponge layer over every uploaded plane (for a slab, its halo
        // planes too), then only the kept planes
        const size_t nvc = (size_t)s->px * s->ny * s->ext_nz;
        DevBuf k1, k2, bmat_full, bd2_full, segcnt_tmp, scan_tmp, total, wtab, flags_ext;
        VIRS_TRY(k1.alloc(nvc * 4, "sponge scratch"));
        VIRS_TRY(k2.alloc(nvc * 4, "sponge scratch"));
        VIRS_TRY(bmat_full.alloc(nvc, "sponge scratch"));
        VIRS_TRY(bd2_full.alloc(nvc * 2, "sponge scratch"));
        if (s->slab) VIRS_TRY(flags_ext.alloc(nvc, "sponge scratch"));
        ClassifyArgs ca{};
        ca.flags_in = s->flags_raw.as<uint8_t>();
        ca.wall_mat = s->wall_mat.as<uint8_t>();
        ca.flags_out = (s->slab ? flags_ext : s->flags).as<uint8_t>();
        ca.bmat_full = bmat_full.as<uint8_t>();
        ca.bd2_full = bd2_full.as<uint16_t>();
        ca.k1 = k1.as<uint32_t>();
        ca.k2 = k2.as<uint32_t>();
        ca.nx = s->nx;
        ca.ny = s->ny;
        ca.nz = s->ext_nz;
        ca.px = s->px;
        ca.W = W;
        VIRS_CUDA(launch_sponge(ca, st));
        k1.release();
        k2.release();
        if (s->slab) {
            // planes are contiguous: one copy per array
            const size_t off = (size_t)s->slab_drop * s->px * s->ny;
            DevBuf bm, bd;
            VIRS_TRY(bm.alloc(s->nvox, "sponge scratch"));
            VIRS_TRY(bd.alloc(s->nvox * 2, "sponge scratch"));
            VIRS_CUDA(cudaMemcpyAsync(s->flags.ptr, flags_ext.as<uint8_t>() + off, s->nvox, cudaMemcpyDeviceToDevice, st));
            VIRS_CUDA(cudaMemcpyAsync(bm.ptr, bmat_full.as<uint8_t>() + off, s->nvox, cudaMemcpyDeviceToDevice, st));
            VIRS_CUDA(cudaMemcpyAsync(bd.ptr, bd2_full.as<uint16_t>() + off, s->nvox * 2, cudaMemcpyDeviceToDevice, st));
            VIRS_CUDA(cudaStreamSynchronize(st));
            std::swap(bmat_full.ptr, bm.ptr);
            std::swap(bmat_full.bytes, bm.bytes);
            std::swap(bd2_full.ptr, bd.ptr);
            std::swap(bd2_full.bytes, bd.bytes);
            flags_ext.release();
        }

        const size_t nseg = (size_t)s->spr * s->ny * s->nz;
        VIRS_TRY(s->code.alloc(s->nvox, "cell codes"));
        VIRS_TRY(s->normals.alloc(s->nvox, "normals"));
        VIRS_TRY(s->bseg.alloc(nseg * 4, "boundary prefix"));
        VIRS_TRY(s->segnz.alloc(nseg, "segment code flags"));
        CodesArgs co{};
        co.flags = s->flags.as<uint8_t>();
        co.code = s->code.as<uint8_t>();
        co.normals = s->normals.as<uint8_t>();
        co.segcnt = s->bseg.as<uint32_t>();
        co.segnz = s->segnz.as<uint8_t>();
        co.nx = s->nx;
        co.ny = s->ny;
        co.nz = s->nz;
        co.px = s->px;
        co.spr = s->spr;
        VIRS_CUDA(launch_codes(co, st));
        {
            DevBuf cnt;
            VIRS_TRY(cnt.alloc(4, "hard-source count"));
            VIRS_CUDA(launch_hard_list(s->code.as<uint8_t>(), s->nvox, cnt.as<uint32_t>(), nullptr, 0, st));
            uint32_t nh = 0;
            VIRS_CUDA(cudaMemcpyAsync(&nh, cnt.ptr, 4, cudaMemcpyDeviceToHost, st));
            VIRS_CUDA(cudaStreamSynchronize(st));
            VIRS_TRY(s->hpos.alloc(std::max<uint32_t>(nh, 1) * 4, "hard-source positions"));
            VIRS_CUDA(cudaMemsetAsync(cnt.ptr, 0, 4, st));
            VIRS_CUDA(launch_hard_list(s->code.as<uint8_t>(), s->nvox, cnt.as<uint32_t>(), s->hpos.as<uint32_t>(), nh,
                                       st));
            VIRS_CUDA(cudaStreamSynchronize(st));
            s->nhpos = nh;
        }
        VIRS_TRY(scan_tmp.alloc(scan_tmp_words(nseg) * 4, "scan scratch"));
        VIRS_TRY(total.alloc(4, "boundary count"));
        VIRS_CUDA(launch_scan(s->bseg.as<uint32_t>(), nseg, scan_tmp.as<uint32_t>(), total.as<uint32_t>(), st));
        uint32_t nb = 0;
        VIRS_CUDA(cudaMemcpyAsync(&nb, total.ptr, 4, cudaMemcpyDeviceToHost, st));
        VIRS_CUDA(cudaStreamSynchronize(st));
        s->nb = nb;

        std::vector<float> wt((size_t)W * W + 1);
        for (int d = 0; d <= W * W; ++d) wt[d] = sponge_weight(W, d);
        VIRS_TRY(wtab.alloc(wt.size() * 4, "sponge weights"));
        VIRS_CUDA(copy_on(s->stream, wtab.ptr, wt.data(), wt.size() * 4, cudaMemcpyHostToDevice));
        VIRS_TRY(s->bidx.alloc(std::max<uint64_t>(nb, 1) * 4, "boundary indices"));
        VIRS_TRY(s->bpos.alloc(std::max<uint64_t>(nb, 1) * 4, "boundary positions"));
        VIRS_TRY(s->bmat.alloc(std::max<uint64_t>(nb, 1), "boundary materials"));
        VIRS_TRY(s->bcode.alloc(std::max<uint64_t>(nb, 1), "boundary codes"));
        VIRS_TRY(s->bnrm.alloc(std::max<uint64_t>(nb, 1), "boundary normals"));
        VIRS_TRY(s->bw.alloc(std::max<uint64_t>(nb, 1) * 4, "boundary weights"));
        VIRS_TRY(s->side.alloc(std::max<uint64_t>(nb, 1) * sizeof(float4), "boundary records"));
        CompactArgs cp{};
        cp.flags = s->flags.as<uint8_t>();
        cp.bseg = s->bseg.as<uint32_t>();
        cp.bmat_full = bmat_full.as<uint8_t>();
        cp.bd2_full = bd2_full.as<uint16_t>();
        cp.wtab = wtab.as<float>();
        cp.bidx = s->bidx.as<uint32_t>();
        cp.bpos = s->bpos.as<uint32_t>();
        cp.bmat = s->bmat.as<uint8_t>();
        cp.code = s->code.as<uint8_t>();
        cp.normals = s->normals.as<uint8_t>();
        cp.bcode = s->bcode.as<uint8_t>();
        cp.bnrm = s->bnrm.as<uint8_t>();
        cp.bw = s->bw.as<float>();
        cp.nx = s->nx;
        cp.ny = s->ny;
        cp.nz = s->nz;
        cp.px = s->px;
        cp.spr = s->spr;
        VIRS_CUDA(launch_compact(cp, st));
        VIRS_CUDA(cudaStreamSynchronize(st));
    }
    s->state.release();
    if (s->filters_set) VIRS_TRY(alloc_states(s));
    s->maps_rows = 0;
    s->zm_rows = s->zm_zc = 0;
    s->zmi_rows = s->zmi_zc = 0;
    s->pm_rows = 0;
    s->pzm_zc = -1;
    s->pl_ok = false;
    s->classified = true;
    VIRS_CUDA(cudaEventRecord(s->done, st));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_flags(const virs_sim *s, uint8_t *out, size_t n)
{
    if (!s || !out) return fail(VIRS_E_ARG, "virs_get_flags: null argument");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    if (n < s->nref) return fail(VIRS_E_ARG, "virs_get_flags: buffer smaller than nx*ny*nz");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    if (s->classified) return d2h_rows(out, s->flags.ptr, 1, s);
    // a slab's kept planes of the uploaded flags
    return d2h_rows(out, s->flags_raw.as<uint8_t>() + (size_t)s->slab_drop * s->px * s->ny, 1, s);
}

VIRS_EXPORT virs_status virs_get_wall_materials(const virs_sim *s, uint8_t *out, size_t n)
{
    if (!s || !out) return fail(VIRS_E_ARG, "virs_get_wall_materials: null argument");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    if (n < s->nref) return fail(VIRS_E_ARG, "virs_get_wall_materials: buffer smaller than nx*ny*nz");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    return d2h_rows(out, s->wall_mat.as<uint8_t>() + (size_t)s->slab_drop * s->px * s->ny, 1, s);
}

VIRS_EXPORT virs_status virs_get_normals(const virs_sim *s, uint8_t *out, size_t n)
{
    if (!s || !out) return fail(VIRS_E_ARG, "virs_get_normals: null argument");
    if (!s->classified) return fail(VIRS_E_STATE, "grid not classified");
    if (n < s->nref) return fail(VIRS_E_ARG, "virs_get_normals: buffer smaller than nx*ny*nz");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    return d2h_rows(out, s->normals.ptr, 1, s);
}

VIRS_EXPORT virs_status virs_get_boundary_indices(const virs_sim *s, uint32_t *out, size_t n)
{
    if (!s || (!out && s->nb)) return fail(VIRS_E_ARG, "virs_get_boundary_indices: null argument");
    if (!s->classified) return fail(VIRS_E_STATE, "grid not classified");
    if (n < s->nb) return fail(VIRS_E_ARG, "virs_get_boundary_indices: buffer smaller than the boundary count");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    if (s->nb) VIRS_CUDA(copy_on(s->stream, out, s->bidx.ptr, s->nb * 4, cudaMemcpyDeviceToHost));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_boundary_materials(const virs_sim *s, uint8_t *mat, float *w, size_t n)
{
    if (!s) return fail(VIRS_E_ARG, "virs_get_boundary_materials: null");
    if (!s->classified) return fail(VIRS_E_STATE, "grid not classified");
    if (n < s->nb) return fail(VIRS_E_ARG, "virs_get_boundary_materials: buffer smaller than the boundary count");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    if (s->nb && mat) VIRS_CUDA(copy_on(s->stream, mat, s->bmat.ptr, s->nb, cudaMemcpyDeviceToHost));
    if (s->nb && w) VIRS_CUDA(copy_on(s->stream, w, s->bw.ptr, s->nb * 4, cudaMemcpyDeviceToHost));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_filters(virs_sim *s, uint32_t nm, uint32_t ns, const float *coeffs)
{
    if (!s || !coeffs) return fail(VIRS_E_ARG, "virs_set_filters: null argument");
    if (nm < 1 || nm > 64 || ns < 1 || ns > 16) return fail(VIRS_E_ARG, "need 1..64 materials and 1..16 sections");
    for (size_t i = 0; i < (size_t)nm * ns * 5; ++i)
        if (!std::isfinite(coeffs[i])) return fail(VIRS_E_ARG, "non-finite filter coefficient");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    VIRS_TRY(s->coef.alloc((size_t)nm * ns * 5 * 4, "filter coefficients"));
    VIRS_CUDA(copy_on(s->stream, s->coef.ptr, coeffs, (size_t)nm * ns * 5 * 4, cudaMemcpyHostToDevice));
    s->nmat = nm;
    s->nsec = ns;
    s->filters_set = true;
    s->graph_dirty = true;
    ++s->gen;
    if (s->classified) VIRS_TRY(alloc_states(s));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_design_highpass(float fs, float fc, float q, float g, float *out5)
{
    if (!out5) return fail(VIRS_E_ARG, "virs_design_highpass: null output");
    rbj_highpass(fs, fc, q, g, out5);
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_design_lowpass(float fs, float fc, float q, float g, float *out5)
{
    if (!out5) return fail(VIRS_E_ARG, "virs_design_lowpass: null output");
    rbj_lowpass(fs, fc, q, g, out5);
    return VIRS_OK;
}

namespace {

// the per-run scale of 16-bit storage: the largest source amplitude maps to
// 2^10, leaving 2^6 of head-room below the FP16 maximum
void choose_scale(virs_sim *s)
{
    if (s->prm.storage == VIRS_STORAGE_F32) {
        s->scale = s->inv_scale = 1.f;
        return;
    }
    if (s->prm.storage_scale > 0.f) {
        s->scale = s->prm.storage_scale;
    } else {
        float peak = 0.f;
        for (float v : s->hard_host) peak = std::max(peak, std::fabs(v));
        peak = std::max(peak, s->sig_peak);
        s->scale = peak > 0.f ? std::exp2f(std::round(std::log2(1024.f / peak))) : 1.f;
    }
    s->inv_scale = 1.f / s->scale;
}

} // namespace

VIRS_EXPORT virs_status virs_set_hard_source(virs_sim *s, const float *v, size_t len)
{
    if (!s || (!v && len)) return fail(VIRS_E_ARG, "virs_set_hard_source: null argument");
    if (len >= (1ull << 32)) return fail(VIRS_E_ARG, "schedule too long");
    for (size_t i = 0; i < len; ++i)
        if (!std::isfinite(v[i])) return fail(VIRS_E_ARG, "non-finite hard source value");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    s->hard_host.assign(v, v + len);
    s->hard.release();
    return VIRS_OK;
}

namespace {
// An audio signal sampled at `rate` read at the simulation times step * dt
// with linear interpolation, following the design written out (commented)
// at simulator_gpu.cu:219-231: float time, float sample index, zero once
// index + 1 reaches the end of the signal.
void audio_to_steps(const float *x, size_t len, float rate, float dt, uint64_t steps, float *out)
{
    for (uint64_t n = 0; n < steps; ++n) {
        const float t = (float)n * dt;
        const float si = t * rate;
        float v = 0.f;
        if (si + 1.f < (float)len) {
            const size_t lo = (size_t)si;
            const float fr = si - (float)lo;
            v = x[lo] + fr * (x[lo + 1] - x[lo]);
        }
        out[n] = v;
    }
}

bool audio_args_ok(const float *x, size_t len, float rate, uint64_t steps)
{
    if (!(rate > 0.f) || !std::isfinite(rate) || steps >= (1ull << 32)) return false;
    for (size_t i = 0; i < len; ++i)
        if (!std::isfinite(x[i])) return false;
    return true;
}
} // namespace

VIRS_EXPORT virs_status virs_set_hard_source_audio(virs_sim *s, const float *samples, size_t len, float sample_rate,
                                                   uint64_t steps)
{
    if (!s || (!samples && len)) return fail(VIRS_E_ARG, "virs_set_hard_source_audio: null argument");
    if (!(s->dt > 0.f)) return fail(VIRS_E_STATE, "no grid: the step size is not known yet");
    if (!audio_args_ok(samples, len, sample_rate, steps))
        return fail(VIRS_E_ARG, "virs_set_hard_source_audio: need a positive sample rate, finite samples, steps < 2^32");
    std::vector<float> v(steps);
    audio_to_steps(samples, len, sample_rate, s->dt, steps, v.data());
    return virs_set_hard_source(s, v.data(), v.size());
}

VIRS_EXPORT virs_status virs_set_sources_audio(virs_sim *s, uint32_t n, const uint64_t *idx, const float *samples,
                                               size_t len, float sample_rate, uint64_t steps)
{
    if (!s || (n && (!idx || (!samples && len)))) return fail(VIRS_E_ARG, "virs_set_sources_audio: null argument");
    if (!(s->dt > 0.f)) return fail(VIRS_E_STATE, "no grid: the step size is not known yet");
    if (!audio_args_ok(samples, (size_t)n * len, sample_rate, steps))
        return fail(VIRS_E_ARG, "virs_set_sources_audio: need a positive sample rate, finite samples, steps < 2^32");
    std::vector<float> sig((size_t)n * steps);
    for (uint32_t i = 0; i < n; ++i)
        audio_to_steps(samples + (size_t)i * len, len, sample_rate, s->dt, steps, sig.data() + (size_t)i * steps);
    return virs_set_sources(s, n, idx, sig.data(), steps);
}

VIRS_EXPORT virs_status virs_set_sources(virs_sim *s, uint32_t n, const uint64_t *idx, const float *sig, size_t len)
{
    if (!s || (n && (!idx || (!sig && len)))) return fail(VIRS_E_ARG, "virs_set_sources: null argument");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    std::vector<uint64_t> dev(n), sorted(idx, idx + n);
    for (uint32_t i = 0; i < n; ++i) {
        if (idx[i] >= s->nref) return fail(VIRS_E_ARG, "source index out of range");
        if (!interior(s, idx[i])) return fail(VIRS_E_ARG, "sources must be interior voxels");
        dev[i] = to_dev(s, idx[i]);
    }
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
        return fail(VIRS_E_ARG, "source voxels must be distinct");
    float peak = 0.f;
    for (size_t i = 0; i < (size_t)n * len; ++i) {
        if (!std::isfinite(sig[i])) return fail(VIRS_E_ARG, "non-finite source sample");
        peak = std::max(peak, std::fabs(sig[i]));
    }
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    s->sig_host.assign(sig, sig + (size_t)n * len);
    s->sig_peak = peak;
    VIRS_TRY(s->src.alloc(std::max<uint32_t>(n, 1) * 8, "source indices"));
    if (n) VIRS_CUDA(copy_on(s->stream, s->src.ptr, dev.data(), n * 8, cudaMemcpyHostToDevice));
    s->nsrc = n;
    s->siglen = len;
    s->src_ref.assign(idx, idx + n);
    s->sig.release();
    s->pl_ok = false;
    s->graph_dirty = true;
    ++s->gen;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_receivers(virs_sim *s, uint32_t n, const uint64_t *idx)
{
    if (!s || (n && !idx)) return fail(VIRS_E_ARG, "virs_set_receivers: null argument");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    std::vector<uint64_t> dev(n);
    for (uint32_t i = 0; i < n; ++i) {
        if (idx[i] >= s->nref) return fail(VIRS_E_ARG, "receiver index out of range");
        dev[i] = to_dev(s, idx[i]);
    }
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    VIRS_TRY(s->rcv.alloc(std::max<uint32_t>(n, 1) * 8, "receiver indices"));
    if (n) VIRS_CUDA(copy_on(s->stream, s->rcv.ptr, dev.data(), n * 8, cudaMemcpyHostToDevice));
    s->nrcv = n;
    s->rcv_ref.assign(idx, idx + n);
    s->ir.release();
    s->ircap = 0;
    s->graph_dirty = true;
    ++s->gen;
    return VIRS_OK;
}

namespace {
virs_status upload_signals(virs_sim *s)
{
    std::vector<float> v(s->sig_host.size());
    for (size_t i = 0; i < v.size(); ++i) v[i] = s->sig_host[i] * s->scale;
    VIRS_TRY(s->sig.alloc(std::max<size_t>(v.size(), 1) * 4, "source signals"));
    if (!v.empty()) VIRS_CUDA(copy_on(s->stream, s->sig.ptr, v.data(), v.size() * 4, cudaMemcpyHostToDevice));
    s->graph_dirty = true;
    ++s->gen;
    return VIRS_OK;
}
} // namespace

VIRS_EXPORT virs_status virs_start_simulation(virs_sim *s, uint64_t steps)
{
    if (!s) return fail(VIRS_E_ARG, "virs_start_simulation: null");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    VIRS_TRY(ready_to_run(s));
    choose_scale(s);
    VIRS_TRY(upload_hard(s));
    VIRS_TRY(upload_signals(s));
    s->ir.release();
    s->ircap = 0;
    VIRS_TRY(ensure_ir(s, std::max<uint64_t>(steps, 1)));
    VIRS_CUDA(zero_on(s->stream, s->field[0].ptr, s->field[0].bytes));
    VIRS_CUDA(zero_on(s->stream, s->field[1].ptr, s->field[1].bytes));
    VIRS_CUDA(zero_on(s->stream, s->state.ptr, s->state.bytes));
    VIRS_CUDA(zero_on(s->stream, s->ctr.ptr, 4));
    if (s->stopbuf.ptr) VIRS_CUDA(zero_on(s->stream, s->stopbuf.ptr, s->stopbuf.bytes));
    s->stopped = false;
    s->slab_open = false;
    s->cur = 0;
    s->steps_done = 0;
    s->out0.clear();
    s->rms_state = 0.f;
    s->fields_valid = true;
    s->drop_graphs();
    VIRS_CUDA(cudaStreamSynchronize(s->stream));
    VIRS_CUDA(cudaEventRecord(s->done, s->stream));
    return VIRS_OK;
}

namespace {
bool started(const virs_sim *s) { return s->sig.ptr && s->hard.ptr && s->ir.ptr; }
} // namespace

VIRS_EXPORT virs_status virs_run(virs_sim *s, uint64_t steps, void *stream)
{
    if (!s) return fail(VIRS_E_ARG, "virs_run: null");
    if (!started(s)) return fail(VIRS_E_STATE, "call virs_start_simulation first");
    if (s->slab_open) return fail(VIRS_E_STATE, "virs_run: a step begun by virs_slab_step_begin has not ended");
    VIRS_TRY(use_device(s));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    if (steps == 0) return VIRS_OK;
    if (s->steps_done + steps >= (1ull << 32)) return fail(VIRS_E_ARG, "step counter would pass 2^32");
    VIRS_CUDA(cudaEventRecord(s->done, s->stream));
    VIRS_CUDA(cudaStreamWaitEvent(st, s->done, 0));
    return run_steps(s, steps, st);
}

namespace {

// lo and hi are adjacent slabs of one grid at the same step
virs_status check_slab_pair(const virs_sim *lo, const virs_sim *hi)
{
    if (!lo->slab || !hi->slab) return fail(VIRS_E_STATE, "slab exchange: a handle is not a slab (virs_set_grid_slab)");
    if (!started(lo) || !started(hi)) return fail(VIRS_E_STATE, "slab exchange: call virs_start_simulation first");
    if (lo->nx != hi->nx || lo->ny != hi->ny || lo->global_nz != hi->global_nz ||
        lo->prm.storage != hi->prm.storage)
        return fail(VIRS_E_ARG, "slab exchange: the slabs belong to different grids or storages");
    if (lo->slab_hi != hi->slab_lo)
        return fail(VIRS_E_ARG, "slab exchange: the slabs are not adjacent (lo owns planes up to " +
                                    std::to_string(lo->slab_hi) + ", hi starts at " + std::to_string(hi->slab_lo) + ")");
    if (lo->steps_done != hi->steps_done || lo->cur != hi->cur)
        return fail(VIRS_E_STATE, "slab exchange: the slabs are not at the same step");
    if (!lo->fields_valid || !hi->fields_valid)
        return fail(VIRS_E_STATE, "slab exchange: the fields were consumed by virs_adjoint");
    return VIRS_OK;
}

// p^n plane k of a slab's current buffer
char *slab_plane(const virs_sim *s, uint64_t k)
{
    return s->field[s->cur].as<char>() + k * (size_t)s->px * s->ny * s->storage_bytes();
}

// each handle pulls its ghost plane from the other on its own stream, after
// the other's last queued work; then each handle's completion event follows
// the copy into its ghost plane
virs_status slab_exchange(virs_sim *lo, virs_sim *hi)
{
    const size_t pb = (size_t)lo->px * lo->ny * lo->storage_bytes();
    VIRS_TRY(use_device(lo));
    VIRS_CUDA(cudaStreamWaitEvent(lo->stream, hi->done, 0));
    VIRS_TRY(use_device(hi));
    VIRS_CUDA(cudaStreamWaitEvent(hi->stream, lo->done, 0));
    VIRS_TRY(use_device(lo));
    VIRS_CUDA(cudaMemcpyAsync(slab_plane(lo, lo->nz - 1), slab_plane(hi, 1), pb, cudaMemcpyDefault, lo->stream));
    VIRS_CUDA(cudaEventRecord(lo->done, lo->stream));
    VIRS_TRY(use_device(hi));
    VIRS_CUDA(cudaMemcpyAsync(slab_plane(hi, 0), slab_plane(lo, lo->nz - 2), pb, cudaMemcpyDefault, hi->stream));
    VIRS_CUDA(cudaEventRecord(hi->done, hi->stream));
    return VIRS_OK;
}

} // namespace

VIRS_EXPORT virs_status virs_slab_exchange(virs_sim *lo, virs_sim *hi)
{
    if (!lo || !hi) return fail(VIRS_E_ARG, "virs_slab_exchange: null argument");
    VIRS_TRY(check_slab_pair(lo, hi));
    return slab_exchange(lo, hi);
}

namespace {

// steps per graph of a slab run (even: the graph leaves every slab's buffer
// parity as it found it)
constexpr int SLAB_GRAPH_STEPS = 16;

// One step of every slab.  Per slab: the interior planes 2 .. nz-3 (they
// read no ghost plane) on the slab's stream; meanwhile, on its exchange
// stream, the pulls of its two ghost planes, after its own and its
// neighbours' previous steps; then, after the pulls, the edge planes 1 and
// nz-2, the boundary pass and the post kernel.  The pulls write the ghost
// planes of p^n, which this step's kernels do not write, and a slab
// overwrites the planes its neighbours pulled from only two steps later,
// after waiting for their previous step, which waited for those pulls.
cudaError_t slab_step(virs_sim *const *slabs, uint32_t n, size_t pb)
{
    cudaError_t e = cudaSuccess;
    for (uint32_t k = 0; k < n && e == cudaSuccess; ++k) {
        virs_sim *s = slabs[k];
        e = cudaSetDevice(s->prm.device);
        const int nz = (int)s->nz;
        if (e == cudaSuccess && nz - 2 > 2) e = launch_stencil_range(s, s->cur, s->stream, 2, nz - 2);
    }
    for (uint32_t k = 0; k < n && e == cudaSuccess; ++k) {
        virs_sim *s = slabs[k];
        e = cudaSetDevice(s->prm.device);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s->xstream, s->done, 0);
        if (e == cudaSuccess && k > 0) {
            e = cudaStreamWaitEvent(s->xstream, slabs[k - 1]->done, 0);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(slab_plane(s, 0), slab_plane(slabs[k - 1], slabs[k - 1]->nz - 2), pb,
                                    cudaMemcpyDefault, s->xstream);
        }
        if (e == cudaSuccess && k + 1 < n) {
            e = cudaStreamWaitEvent(s->xstream, slabs[k + 1]->done, 0);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(slab_plane(s, s->nz - 1), slab_plane(slabs[k + 1], 1), pb, cudaMemcpyDefault,
                                    s->xstream);
        }
        if (e == cudaSuccess) e = cudaEventRecord(s->xdone, s->xstream);
    }
    for (uint32_t k = 0; k < n && e == cudaSuccess; ++k) {
        virs_sim *s = slabs[k];
        e = cudaSetDevice(s->prm.device);
        const int nz = (int)s->nz, par = s->cur;
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s->stream, s->xdone, 0);
        if (e == cudaSuccess) e = launch_stencil_range(s, par, s->stream, 1, 2);
        if (e == cudaSuccess && nz - 2 > 1) e = launch_stencil_range(s, par, s->stream, nz - 2, nz - 1);
        if (e == cudaSuccess) e = launch_boundary(s->prm.storage, step_args(s, par), BND_UPDATE, s->stream);
        if (e == cudaSuccess) e = launch_post(s->prm.storage, post_args(s, par), s->stream);
        if (e == cudaSuccess) {
            s->cur ^= 1;
            s->steps_done += 1;
            e = cudaEventRecord(s->done, s->stream);
        }
    }
    return e;
}

// events that live for one call
struct EventSet {
    std::vector<cudaEvent_t> ev;
    ~EventSet()
    {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    cudaError_t make(cudaEvent_t *out)
    {
        const cudaError_t e = cudaEventCreateWithFlags(out, cudaEventDisableTiming);
        if (e == cudaSuccess) ev.push_back(*out);
        return e;
    }
};

// SLAB_GRAPH_STEPS steps of all slabs (one device) captured in one graph
// from the first slab's stream: the other streams join the capture through
// an event recorded on it and leave it through events it waits for; each
// slab records its completion event inside the capture before any wait on
// it.  The steps are enqueued as slab_step does; the handles' step state is
// put back after the capture (the graph's launches advance it), and so are
// their events.
virs_status slab_graph(virs_sim *const *slabs, uint32_t n, size_t pb, cudaGraphExec_t *exec)
{
    VIRS_TRY(use_device(slabs[0]));
    cudaStream_t o = slabs[0]->stream;
    EventSet evs;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join(2 * n, nullptr);
    VIRS_CUDA(evs.make(&fork));
    for (auto &j : join) VIRS_CUDA(evs.make(&j));
    std::vector<int> cur(n);
    std::vector<uint64_t> done(n);
    for (uint32_t k = 0; k < n; ++k) {
        cur[k] = slabs[k]->cur;
        done[k] = slabs[k]->steps_done;
    }
    VIRS_CUDA(cudaStreamBeginCapture(o, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaEventRecord(fork, o);
    for (uint32_t k = 0; k < n && e == cudaSuccess; ++k) {
        virs_sim *s = slabs[k];
        if (k > 0) e = cudaStreamWaitEvent(s->stream, fork, 0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s->xstream, fork, 0);
        if (e == cudaSuccess) e = cudaEventRecord(s->done, s->stream);
    }
    for (int i = 0; i < SLAB_GRAPH_STEPS && e == cudaSuccess; ++i) e = slab_step(slabs, n, pb);
    for (uint32_t k = 0; k < n && e == cudaSuccess; ++k) {
        virs_sim *s = slabs[k];
        if (k > 0) {
            e = cudaEventRecord(join[2 * k], s->stream);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(o, join[2 * k], 0);
        }
        if (e == cudaSuccess) e = cudaEventRecord(join[2 * k + 1], s->xstream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(o, join[2 * k + 1], 0);
    }
    for (uint32_t k = 0; k < n; ++k) {
        slabs[k]->cur = cur[k];
        slabs[k]->steps_done = done[k];
    }
    cudaSetDevice(slabs[0]->prm.device);
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(o, &g);
    if (e == cudaSuccess) e = ee;
    // the events recorded during the capture stand for graph nodes: record
    // them again on their streams, whose queued work the capture left as it
    // was
    for (uint32_t k = 0; k < n; ++k) {
        const cudaError_t er = cudaEventRecord(slabs[k]->done, slabs[k]->stream);
        const cudaError_t ex = cudaEventRecord(slabs[k]->xdone, slabs[k]->xstream);
        if (e == cudaSuccess) e = er != cudaSuccess ? er : ex;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "slab step graph");
    }
    return VIRS_OK;
}

// `times` launches of the graph on the first slab's stream, after every
// slab's queued work; every slab's stream then follows the last launch
virs_status slab_graph_run(virs_sim *const *slabs, uint32_t n, cudaGraphExec_t exec, uint64_t times)
{
    VIRS_TRY(use_device(slabs[0]));
    cudaStream_t o = slabs[0]->stream;
    EventSet evs;
    cudaEvent_t after = nullptr;
    VIRS_CUDA(evs.make(&after));
    for (uint32_t k = 1; k < n; ++k) VIRS_CUDA(cudaStreamWaitEvent(o, slabs[k]->done, 0));
    for (uint64_t r = 0; r < times; ++r) VIRS_CUDA(cudaGraphLaunch(exec, o));
    VIRS_CUDA(cudaEventRecord(after, o));
    for (uint32_t k = 0; k < n; ++k) {
        virs_sim *s = slabs[k];
        if (k > 0) VIRS_CUDA(cudaStreamWaitEvent(s->stream, after, 0));
        VIRS_CUDA(cudaStreamWaitEvent(s->xstream, after, 0));
        VIRS_CUDA(cudaEventRecord(s->done, s->stream));
        s->steps_done += times * SLAB_GRAPH_STEPS;
    }
    return VIRS_OK;
}

} // namespace

VIRS_EXPORT virs_status virs_slab_run(virs_sim *const *slabs, uint32_t n, uint64_t steps)
{
    if (!slabs || n == 0) return fail(VIRS_E_ARG, "virs_slab_run: no slabs");
    for (uint32_t k = 0; k < n; ++k) {
        if (!slabs[k]) return fail(VIRS_E_ARG, "virs_slab_run: null slab");
        if (slabs[k]->slab_open)
            return fail(VIRS_E_STATE, "virs_slab_run: a step begun by virs_slab_step_begin has not ended");
        if (slabs[k]->stop_rule) return fail(VIRS_E_STATE, "virs_slab_run: the device stop rule is not for slabs");
    }
    if (n == 1) {
        const virs_sim *s = slabs[0];
        if (!s->slab || !started(s)) return fail(VIRS_E_STATE, "virs_slab_run: a started slab handle is needed");
        if (!s->fields_valid) return fail(VIRS_E_STATE, "virs_slab_run: the fields were consumed by virs_adjoint");
    }
    for (uint32_t k = 0; k + 1 < n; ++k) VIRS_TRY(check_slab_pair(slabs[k], slabs[k + 1]));
    if (slabs[0]->slab_lo != 1 || slabs[n - 1]->slab_hi != slabs[0]->global_nz - 1)
        return fail(VIRS_E_ARG, "virs_slab_run: the slabs must cover the grid's interior planes, in order");
    if (slabs[0]->steps_done + steps >= (1ull << 32)) return fail(VIRS_E_ARG, "step counter would pass 2^32");
    for (uint32_t k = 0; k < n; ++k) {
        virs_sim *s = slabs[k];
        VIRS_TRY(use_device(s));
        if (s->stop_rule && s->stopped) return fail(VIRS_E_STATE, "virs_slab_run: the stop rule fired");
        VIRS_TRY(ready_to_run(s));
        VIRS_TRY(ensure_ir(s, s->steps_done + steps));
        if (s->depth > 0 && zero_masks_useful(s) && s->nz > 5 &&
            (s->zmi_rows != s->tile_rows || s->zmi_zc != eff_planes(s))) {
            s->zmi_rows = s->zmi_zc = 0;
            VIRS_TRY(build_zero_masks(s, s->tile_rows, eff_planes(s), s->zmask_in, 2, s->nz - 2));
            s->zmi_rows = s->tile_rows;
            s->zmi_zc = eff_planes(s);
        }
        if (!s->xstream) VIRS_CUDA(cudaStreamCreateWithFlags(&s->xstream, cudaStreamNonBlocking));
        if (!s->xdone) VIRS_CUDA(cudaEventCreateWithFlags(&s->xdone, cudaEventDisableTiming));
    }
    const size_t pb = (size_t)slabs[0]->px * slabs[0]->ny * slabs[0]->storage_bytes();
    bool one_device = true;
    for (uint32_t k = 1; k < n; ++k) one_device = one_device && slabs[k]->prm.device == slabs[0]->prm.device;
    uint64_t i = 0;
    if (one_device && n > 1 && steps >= SLAB_GRAPH_STEPS) {
        std::unique_ptr<SlabGraph> &c = slabs[0]->slab_graph;
        bool same = c && c->mem.size() == n;
        for (uint32_t k = 0; same && k < n; ++k)
            same = c->mem[k] == slabs[k] && c->id[k] == slabs[k]->id && c->gen[k] == slabs[k]->gen;
        if (!same) {
            c.reset(new SlabGraph);
            for (uint32_t k = 0; k < n; ++k) {
                c->mem.push_back(slabs[k]);
                c->id.push_back(slabs[k]->id);
                c->gen.push_back(slabs[k]->gen);
            }
        }
        const int par = slabs[0]->cur;
        if (!c->exec[par]) VIRS_TRY(slab_graph(slabs, n, pb, &c->exec[par]));
        VIRS_TRY(slab_graph_run(slabs, n, c->exec[par], steps / SLAB_GRAPH_STEPS));
        i = steps / SLAB_GRAPH_STEPS * SLAB_GRAPH_STEPS;
    }
    for (; i < steps; ++i) VIRS_CUDA(slab_step(slabs, n, pb));
    return VIRS_OK;
}

namespace {
// a slab handle ready for one more step of the split form
virs_status slab_step_ready(virs_sim *s, const char *who)
{
    if (!s->slab || !started(s)) return fail(VIRS_E_STATE, std::string(who) + ": a started slab handle is needed");
    if (!s->fields_valid) return fail(VIRS_E_STATE, std::string(who) + ": the fields were consumed by virs_adjoint");
    if (s->stop_rule) return fail(VIRS_E_STATE, std::string(who) + ": the device stop rule is not for slabs");
    if (s->steps_done + 1 >= (1ull << 32)) return fail(VIRS_E_ARG, "step counter would pass 2^32");
    VIRS_TRY(use_device(s));
    VIRS_TRY(ready_to_run(s));
    VIRS_TRY(ensure_ir(s, s->steps_done + 1));
    if (s->depth > 0 && zero_masks_useful(s) && s->nz > 5 &&
        (s->zmi_rows != s->tile_rows || s->zmi_zc != eff_planes(s))) {
        s->zmi_rows = s->zmi_zc = 0;
        VIRS_TRY(build_zero_masks(s, s->tile_rows, eff_planes(s), s->zmask_in, 2, s->nz - 2));
        s->zmi_rows = s->tile_rows;
        s->zmi_zc = eff_planes(s);
    }
    return VIRS_OK;
}
} // namespace

VIRS_EXPORT virs_status virs_slab_step_begin(virs_sim *s, void *stream)
{
    if (!s) return fail(VIRS_E_ARG, "virs_slab_step_begin: null");
    if (s->slab_open) return fail(VIRS_E_STATE, "virs_slab_step_begin: the step begun before has not ended");
    VIRS_TRY(slab_step_ready(s, "virs_slab_step_begin"));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    VIRS_CUDA(cudaStreamWaitEvent(st, s->done, 0));
    const int nz = (int)s->nz;
    if (nz - 2 > 2) VIRS_CUDA(launch_stencil_range(s, s->cur, st, 2, nz - 2));
    s->slab_open = true;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_slab_step_end(virs_sim *s, void *stream)
{
    if (!s) return fail(VIRS_E_ARG, "virs_slab_step_end: null");
    if (!s->slab_open) return fail(VIRS_E_STATE, "virs_slab_step_end: no step begun (virs_slab_step_begin)");
    VIRS_TRY(use_device(s));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    const int nz = (int)s->nz, par = s->cur;
    s->slab_open = false;
    VIRS_CUDA(launch_stencil_range(s, par, st, 1, 2));
    if (nz - 2 > 1) VIRS_CUDA(launch_stencil_range(s, par, st, nz - 2, nz - 1));
    VIRS_CUDA(launch_boundary(s->prm.storage, step_args(s, par), BND_UPDATE, st));
    VIRS_CUDA(launch_post(s->prm.storage, post_args(s, par), st));
    s->cur ^= 1;
    s->steps_done += 1;
    VIRS_CUDA(cudaEventRecord(s->done, st));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_synchronize(virs_sim *s)
{
    if (!s) return fail(VIRS_E_ARG, "virs_synchronize: null");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    return check_err(s);
}

VIRS_EXPORT virs_status virs_run_host(virs_sim *s, uint64_t steps, const float *signal, float *ir_out, void *stream)
{
    if (!s) return fail(VIRS_E_ARG, "virs_run_host: null");
    if (!started(s)) return fail(VIRS_E_STATE, "call virs_start_simulation first");
    VIRS_TRY(use_device(s));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    const uint64_t first = s->steps_done;
    VIRS_CUDA(cudaEventRecord(s->done, s->stream));
    VIRS_CUDA(cudaStreamWaitEvent(st, s->done, 0));
    if (signal && s->nsrc) {
        if (first + steps > s->siglen)
            return fail(VIRS_E_ARG, "virs_run_host: source signals were set for fewer steps than requested");
        // the host samples of these steps, scaled like the stored field
        const float *src = signal;
        std::vector<float> scaled;
        if (s->scale != 1.f) {
            scaled.assign(signal, signal + (size_t)s->nsrc * steps);
            for (float &v : scaled) v *= s->scale;
            src = scaled.data();
        }
        VIRS_CUDA(cudaMemcpy2DAsync(s->sig.as<float>() + first, s->siglen * 4, src, steps * 4, steps * 4, s->nsrc,
                                    cudaMemcpyHostToDevice, st));
    }
    VIRS_TRY(run_steps(s, steps, st));
    if (ir_out && s->nrcv)
        VIRS_CUDA(cudaMemcpy2DAsync(ir_out, steps * 4, s->ir.as<float>() + first, s->ircap * 4, steps * 4, s->nrcv,
                                    cudaMemcpyDeviceToHost, st));
    VIRS_CUDA(cudaStreamSynchronize(st));
    return check_err(s);
}

VIRS_EXPORT virs_status virs_step(virs_sim *s, uint32_t step, int *keep_going, float *sample)
{
    if (!s) return fail(VIRS_E_ARG, "virs_step: null");
    if (s->stop_rule)
        return fail(VIRS_E_STATE, "virs_step applies the stop rule on the host: disable the device rule (virs_set_stop_rule)");
    if (!started(s)) return fail(VIRS_E_STATE, "call virs_start_simulation first");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    VIRS_TRY(ready_to_run(s));
    VIRS_TRY(ensure_ir(s, (uint64_t)step + 1));
    cudaStream_t st = s->stream;
    // the reference uploads the source value every step (simulator_gpu.cu:250-258)
    VIRS_CUDA(cudaMemcpyAsync(s->ctr.ptr, &step, 4, cudaMemcpyHostToDevice, st));
    cudaError_t e = enqueue_step(s, s->cur, st);
    if (e != cudaSuccess) return cuda_fail(e, "step launch");
    s->cur ^= 1;
    s->steps_done = std::max<uint64_t>(s->steps_done, (uint64_t)step + 1);
    float v = 0.f;
    if (s->nrcv) VIRS_CUDA(cudaMemcpyAsync(&v, s->ir.as<float>() + step, 4, cudaMemcpyDeviceToHost, st));
    VIRS_CUDA(cudaStreamSynchronize(st));
    VIRS_CUDA(cudaEventRecord(s->done, st));
    VIRS_TRY(check_err(s));
    if (sample) *sample = v;
    if (!std::isfinite(v)) return fail(VIRS_E_UNSTABLE, "receiver sample is not finite at step " + std::to_string(step));
    if (s->out0.size() <= step) s->out0.resize((size_t)step + 1, 0.f);
    s->out0[step] = v;
    bool go = true;
    // simulator_gpu.cu:303-330
    constexpr uint32_t RMS_SIZE = 100, MIN_RMS_CHECK_STEP = 3000;
    if (step > MIN_RMS_CHECK_STEP) {
        float sum = 0.0f;
        for (uint32_t i = step - RMS_SIZE; i < step; ++i) sum += s->out0[i] * s->out0[i];
        float rms = std::sqrt(sum / (float)RMS_SIZE);
        if (step == MIN_RMS_CHECK_STEP + 1) {
            s->rms_state = rms;
        } else {
            const float g = 0.00008f;
            const float vout = (g * rms + s->rms_state) / (g + 1.f);
            s->rms_state = 2.f * vout - s->rms_state;
            rms = vout;
        }
        if (rms < 0.0009f) go = false;
    }
    if (keep_going) *keep_going = go ? 1 : 0;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_stop_rule(virs_sim *s, int enable)
{
    if (!s) return fail(VIRS_E_ARG, "virs_set_stop_rule: null");
    if (enable != 0 && enable != 1) return fail(VIRS_E_ARG, "virs_set_stop_rule: enable must be 0 or 1");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    if (enable && !s->stopbuf.ptr) VIRS_TRY(s->stopbuf.alloc(4 * sizeof(uint32_t), "stop rule state"));
    if (s->stopbuf.ptr) VIRS_CUDA(zero_on(s->stream, s->stopbuf.ptr, s->stopbuf.bytes));
    s->stop_rule = enable != 0;
    s->stopped = false;
    s->drop_graphs();
    ++s->gen;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_stop(const virs_sim *s, int *stopped, uint64_t *stop_step)
{
    if (!s || !stopped || !stop_step) return fail(VIRS_E_ARG, "virs_get_stop: null argument");
    *stopped = s->stopped ? 1 : 0;
    *stop_step = s->stopped ? s->stop_step : 0;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_ir(const virs_sim *s, uint64_t first, uint64_t steps, float *out)
{
    if (!s || (!out && steps && s->nrcv)) return fail(VIRS_E_ARG, "virs_get_ir: null argument");
    if (first + steps > s->steps_done) return fail(VIRS_E_ARG, "virs_get_ir: steps not run yet");
    if (!s->nrcv || !steps) return VIRS_OK;
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    VIRS_TRY(check_err(const_cast<virs_sim *>(s)));
    VIRS_CUDA(copy2d_on(s->stream, out, steps * 4, s->ir.as<float>() + first, s->ircap * 4, steps * 4, s->nrcv,
                           cudaMemcpyDeviceToHost));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_postprocess_ir(virs_sim *s, double rate, const double *sos, uint32_t ns, int normalize,
                                            float *out, uint64_t capacity, uint64_t *out_len)
{
    if (!s || !out_len || (ns && !sos)) return fail(VIRS_E_ARG, "virs_postprocess_ir: null argument");
    if (!(rate > 0.0) || !std::isfinite(rate)) return fail(VIRS_E_ARG, "virs_postprocess_ir: rate must be > 0");
    if (ns > 32) return fail(VIRS_E_ARG, "virs_postprocess_ir: at most 32 sections");
    if (!(s->dt > 0.f)) return fail(VIRS_E_STATE, "virs_postprocess_ir: no grid");
    const uint64_t steps = s->steps_done;
    const uint64_t len = (uint64_t)(rate * ((double)steps * (double)s->dt));
    *out_len = len;
    if (!out || !len || !s->nrcv) return VIRS_OK;
    if (capacity < len) return fail(VIRS_E_ARG, "virs_postprocess_ir: capacity smaller than the output length");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    VIRS_TRY(check_err(s));
    // the simulation rate as the reference forms it: 1.f / dt in float
    const double sim_rate = (double)(1.f / s->dt);
    cudaStream_t st = s->stream;
    DevBuf dsos, filt, res;
    const float *src = s->ir.as<float>();
    uint64_t stride = s->ircap;
    if (ns) {
        VIRS_TRY(dsos.alloc((size_t)ns * 6 * sizeof(double), "post-processing sections"));
        VIRS_TRY(filt.alloc((size_t)s->nrcv * steps * sizeof(float), "filtered receiver traces"));
        VIRS_CUDA(cudaMemcpyAsync(dsos.ptr, sos, (size_t)ns * 6 * sizeof(double), cudaMemcpyHostToDevice, st));
        VIRS_CUDA(launch_ir_sos(src, stride, steps, dsos.as<double>(), (int)ns, filt.as<float>(), steps, s->nrcv, st));
        src = filt.as<float>();
        stride = steps;
    }
    VIRS_TRY(res.alloc((size_t)s->nrcv * len * sizeof(float), "resampled receiver traces"));
    VIRS_CUDA(launch_ir_resample(src, stride, steps, sim_rate, (float)rate, res.as<float>(), len, normalize ? 1 : 0,
                                 s->nrcv, st));
    VIRS_CUDA(cudaMemcpyAsync(out, res.ptr, (size_t)s->nrcv * len * sizeof(float), cudaMemcpyDeviceToHost, st));
    VIRS_CUDA(cudaStreamSynchronize(st));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_postprocess_ir_sinc(virs_sim *s, double rate, uint32_t half_taps, double beta,
                                                 double cutoff, int normalize, float *out, uint64_t capacity,
                                                 uint64_t *out_len)
{
    if (!s || !out_len) return fail(VIRS_E_ARG, "virs_postprocess_ir_sinc: null argument");
    if (!(rate > 0.0) || !std::isfinite(rate)) return fail(VIRS_E_ARG, "virs_postprocess_ir_sinc: rate must be > 0");
    if (half_taps < 1 || half_taps > 4096) return fail(VIRS_E_ARG, "virs_postprocess_ir_sinc: half_taps must be 1..4096");
    if (!(beta >= 0.0) || !(beta <= 50.0)) return fail(VIRS_E_ARG, "virs_postprocess_ir_sinc: beta must be 0..50");
    if (!(cutoff > 0.0) || !(cutoff <= 1.0)) return fail(VIRS_E_ARG, "virs_postprocess_ir_sinc: cutoff must be in (0, 1]");
    if (!(s->dt > 0.f)) return fail(VIRS_E_STATE, "virs_postprocess_ir_sinc: no grid");
    const uint64_t steps = s->steps_done;
    const uint64_t len = (uint64_t)(rate * ((double)steps * (double)s->dt));
    *out_len = len;
    if (!out || !len || !s->nrcv) return VIRS_OK;
    if (capacity < len) return fail(VIRS_E_ARG, "virs_postprocess_ir_sinc: capacity smaller than the output length");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    VIRS_TRY(check_err(s));
    cudaStream_t st = s->stream;
    DevBuf res, peak;
    VIRS_TRY(res.alloc((size_t)s->nrcv * len * sizeof(float), "resampled receiver traces"));
    if (normalize) VIRS_TRY(peak.alloc((size_t)s->nrcv * sizeof(uint32_t), "receiver peaks"));
    VIRS_CUDA(launch_ir_sinc(s->ir.as<float>(), s->ircap, steps, 1.0 / (double)s->dt, rate, (int)half_taps, beta,
                             cutoff, res.as<float>(), len, normalize ? peak.as<uint32_t>() : nullptr, s->nrcv, st));
    VIRS_CUDA(cudaMemcpyAsync(out, res.ptr, (size_t)s->nrcv * len * sizeof(float), cudaMemcpyDeviceToHost, st));
    VIRS_CUDA(cudaStreamSynchronize(st));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_pressure(const virs_sim *s, float *cur, float *prev, size_t n)
{
    if (!s || !cur) return fail(VIRS_E_ARG, "virs_get_pressure: null argument");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    if (n < s->nref) return fail(VIRS_E_ARG, "virs_get_pressure: buffer smaller than nx*ny*nz");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    float *outs[2] = {cur, prev};
    for (int k = 0; k < 2; ++k) {
        if (!outs[k]) continue;
        const DevBuf &f = s->field[s->cur ^ k];
        if (s->prm.storage == VIRS_STORAGE_F32) {
            VIRS_TRY(d2h_rows(outs[k], f.ptr, 4, s));
        } else {
            DevBuf tmp;
            VIRS_TRY(tmp.alloc(s->nref * 4, "pressure export"));
            VIRS_CUDA(launch_pack(s->prm.storage, f.ptr, tmp.as<float>(), s->nx, s->ny, s->nz, s->px, s->inv_scale,
                                  s->stream));
            VIRS_CUDA(cudaMemcpyAsync(outs[k], tmp.ptr, s->nref * 4, cudaMemcpyDeviceToHost, s->stream));
            VIRS_CUDA(cudaStreamSynchronize(s->stream));
        }
    }
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_pressure(virs_sim *s, const float *cur, const float *prev, size_t n)
{
    if (!s || !cur) return fail(VIRS_E_ARG, "virs_set_pressure: null argument");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    if (n < s->nref) return fail(VIRS_E_ARG, "virs_set_pressure: buffer smaller than nx*ny*nz");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    const float *ins[2] = {cur, prev};
    for (int k = 0; k < 2; ++k) {
        DevBuf &f = s->field[s->cur ^ k];
        if (!ins[k]) {
            VIRS_CUDA(zero_on(s->stream, f.ptr, f.bytes));
            continue;
        }
        if (s->prm.storage == VIRS_STORAGE_F32) {
            VIRS_TRY(h2d_rows(f.ptr, ins[k], 4, s));
        } else {
            DevBuf tmp;
            VIRS_TRY(tmp.alloc(s->nref * 4, "pressure import"));
            VIRS_CUDA(copy_on(s->stream, tmp.ptr, ins[k], s->nref * 4, cudaMemcpyHostToDevice));
            VIRS_CUDA(launch_unpack(s->prm.storage, tmp.as<float>(), f.ptr, s->nx, s->ny, s->nz, s->px, s->scale,
                                    s->stream));
            VIRS_CUDA(cudaStreamSynchronize(s->stream));
        }
    }
    VIRS_CUDA(cudaEventRecord(s->done, s->stream));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_init_pressure_sphere(virs_sim *s, uint64_t x, uint64_t y, uint64_t z, uint64_t r,
                                                  float value, int init)
{
    if (!s) return fail(VIRS_E_ARG, "virs_init_pressure_sphere: null");
    if (!s->has_grid) return fail(VIRS_E_STATE, "no grid");
    // vectorspace.cpp / simulator_cpu.cpp:86-90 range checks
    if (x >= s->nx || y >= s->ny || z >= s->nz) return fail(VIRS_E_ARG, "initPressureSphere: position out of range");
    if (r > s->nx / 2 || r > s->ny / 2 || r > s->nz / 2)
        return fail(VIRS_E_ARG, "initPressureSphere: radius exceeds half of grid dimensions");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    VIRS_CUDA(launch_sphere(s->prm.storage, s->field[s->cur].ptr, s->nx, s->ny, s->nz, s->px, x, y, z, r,
                            value * s->scale, init, s->stream));
    VIRS_CUDA(cudaEventRecord(s->done, s->stream));
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_energy(virs_sim *s, double *out)
{
    if (!s || !out) return fail(VIRS_E_ARG, "virs_energy: null argument");
    if (!s->classified) return fail(VIRS_E_STATE, "grid not classified");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    const int nblocks = 148 * 8;
    if (!s->energy_partial.ptr) VIRS_TRY(s->energy_partial.alloc((nblocks + 1) * sizeof(double), "energy partials"));
    const double lambda2 = (double)s->c2dt2 * (double)s->inv_h2;
    const double is2 = (double)s->inv_scale * (double)s->inv_scale;
    VIRS_CUDA(launch_energy(s->prm.storage, s->field[s->cur].ptr, s->field[s->cur ^ 1].ptr, s->code.as<uint8_t>(),
                            s->nx, s->ny, s->nz, s->px, lambda2, is2, s->energy_partial.as<double>(), nblocks,
                            s->stream));
    VIRS_CUDA(cudaMemcpyAsync(out, s->energy_partial.as<double>() + nblocks, sizeof(double), cudaMemcpyDeviceToHost,
                              s->stream));
    VIRS_CUDA(cudaStreamSynchronize(s->stream));
    if (!std::isfinite(*out)) return fail(VIRS_E_UNSTABLE, "energy is not finite");
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_timing(virs_sim *s, int enable)
{
    if (!s) return fail(VIRS_E_ARG, "virs_set_timing: null");
    s->timing = enable != 0;
    s->t_ms = s->t_bms = 0;
    s->t_steps = s->t_launch = 0;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_timing(virs_sim *s, virs_timing *o)
{
    if (!s || !o) return fail(VIRS_E_ARG, "virs_get_timing: null argument");
    o->step_kernel_ms = s->t_ms;
    o->boundary_kernel_ms = s->t_bms;
    o->step_launches = s->t_steps;
    o->kernel_launches = s->t_launch;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_tiling(virs_sim *s, int rows, int planes, int depth)
{
    if (!s) return fail(VIRS_E_ARG, "virs_set_tiling: null");
    if (rows != 0 && rows != 4 && rows != 8 && rows != 16) return fail(VIRS_E_ARG, "tile rows must be 4, 8 or 16");
    if (planes < 0 || planes > 4096) return fail(VIRS_E_ARG, "planes per block must be 0..4096");
    if (depth < -1 || depth > 3) return fail(VIRS_E_ARG, "pipeline depth must be -1 (default), 0 (no TMA) or 1..3");
    VIRS_TRY(wait_done(s));
    s->tile_rows = rows ? rows : 8;
    s->zc = planes;
    s->depth = depth < 0 ? 2 : depth;
    s->maps_rows = 0;
    s->drop_graphs();
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_time_blocking(virs_sim *s, int steps_per_pass, int tile_rows, int planes)
{
    if (!s) return fail(VIRS_E_ARG, "virs_set_time_blocking: null");
    if (steps_per_pass != 1 && steps_per_pass != 2) return fail(VIRS_E_ARG, "steps per pass must be 1 or 2");
    if (tile_rows != 0 && tile_rows != 12 && tile_rows != 14 && tile_rows != 16 && tile_rows != 32)
        return fail(VIRS_E_ARG, "two-step tile rows must be 12, 14, 16 or 32");
    if (planes < 0 || planes > 4096) return fail(VIRS_E_ARG, "planes per block must be 0..4096");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    s->pair_steps = steps_per_pass;
    s->pair_rows = tile_rows ? tile_rows : 14;
    s->pair_zc = planes;
    s->pm_rows = 0;
    s->pair_nomem = false;
    if (steps_per_pass == 1) {
        s->spare[0].release();
        s->spare[1].release();
        s->plist.release();
        s->nplist = 0;
        s->pl_ok = false;
    }
    s->drop_graphs();
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_set_rounding(virs_sim *s, int mode)
{
    if (!s) return fail(VIRS_E_ARG, "virs_set_rounding: null");
    if (mode != VIRS_ROUND_NEAREST && mode != VIRS_ROUND_STOCHASTIC)
        return fail(VIRS_E_ARG, "rounding must be VIRS_ROUND_NEAREST or VIRS_ROUND_STOCHASTIC");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    s->rounding = mode;
    s->drop_graphs();
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_time_blocking(const virs_sim *s, int *steps_per_pass, int *tile_rows, int *planes,
                                               int *active)
{
    if (!s || !steps_per_pass || !tile_rows || !planes || !active)
        return fail(VIRS_E_ARG, "virs_get_time_blocking: null argument");
    *steps_per_pass = s->pair_steps;
    *tile_rows = s->pair_rows;
    *planes = s->pair_zc;
    *active = pair_on(s) ? 1 : 0;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_check_bounded_wait(virs_sim *s, uint32_t limit)
{
    if (!s) return fail(VIRS_E_ARG, "virs_check_bounded_wait: null");
    if (limit == 0 || limit > (1u << 20)) return fail(VIRS_E_ARG, "limit must be 1..2^20");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    if (!s->err.ptr) VIRS_TRY(s->err.alloc(sizeof(int), "error flag"));
    VIRS_CUDA(launch_wait_probe(s->err.as<int>(), limit, s->stream));
    VIRS_CUDA(cudaStreamSynchronize(s->stream));
    return check_err(s);
}

namespace {

// best tiling per (device, storage, nx, ny, nz), filled by virs_autotune
struct TuneKey {
    int dev, storage;
    uint32_t nx, ny, nz;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(dev, storage, nx, ny, nz) < std::tie(o.dev, o.storage, o.nx, o.ny, o.nz);
    }
};
// the single-step tiling, and the two-step settings when those won
struct TunePick {
    virs_tiling t{};
    int pair_steps = 1, pair_rows = 14, pair_zc = 0;
};
std::mutex g_tune_mu;
std::map<TuneKey, TunePick> g_tune;

virs_status reset_state(virs_sim *s)
{
    VIRS_CUDA(cudaMemsetAsync(s->field[0].ptr, 0, s->field[0].bytes, s->stream));
    VIRS_CUDA(cudaMemsetAsync(s->field[1].ptr, 0, s->field[1].bytes, s->stream));
    VIRS_CUDA(cudaMemsetAsync(s->state.ptr, 0, s->state.bytes, s->stream));
    VIRS_CUDA(cudaMemsetAsync(s->ctr.ptr, 0, 4, s->stream));
    if (s->stopbuf.ptr) VIRS_CUDA(cudaMemsetAsync(s->stopbuf.ptr, 0, s->stopbuf.bytes, s->stream));
    s->stopped = false;
    if (s->ir.ptr) VIRS_CUDA(cudaMemsetAsync(s->ir.ptr, 0, s->ir.bytes, s->stream));
    VIRS_CUDA(cudaStreamSynchronize(s->stream));
    s->cur = 0;
    s->steps_done = 0;
    s->out0.clear();
    s->rms_state = 0.f;
    return VIRS_OK;
}

} // namespace

VIRS_EXPORT virs_status virs_autotune(virs_sim *s, uint32_t trial_steps, virs_tiling *best)
{
    if (!s) return fail(VIRS_E_ARG, "virs_autotune: null");
    if (!started(s)) return fail(VIRS_E_STATE, "call virs_start_simulation first");
    if (s->steps_done != 0) return fail(VIRS_E_STATE, "virs_autotune must run before the first step");
    if (trial_steps == 0 || trial_steps > 1000) return fail(VIRS_E_ARG, "trial_steps must be 1..1000");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    const TuneKey key{s->prm.device, s->prm.storage, s->nx, s->ny, s->nz};
    TunePick pick{};
    bool cached = false;
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            pick = it->second;
            cached = true;
        }
    }
    if (!cached) {
        // two-step trials: at least two groups of four steps each
        const uint32_t quads = std::max<uint32_t>(2, (trial_steps + 3) / 4);
        VIRS_TRY(ensure_ir(s, std::max<uint64_t>(2ull * trial_steps, 4ull * quads + 4) + 2));
        s->pair_steps = 1;
        cudaEvent_t e0, e1;
        VIRS_CUDA(cudaEventCreate(&e0));
        VIRS_CUDA(cudaEventCreate(&e1));
        float best_ms = 1e30f;
        // Every candidate is timed twice, in forward and then reverse order:
        // a sustained load brings the GPU to its power cap within about a
        // second, which would favour the candidates timed first.
        struct Cand {
            int d, r, pl;
        };
        std::vector<Cand> sc;
        for (int d : {1, 2, 3})
            for (int r : {4, 8, 16})
                for (int pl : {8, 16, 32, 64}) sc.push_back({d, r, pl});
        virs_status st = VIRS_OK;
        for (size_t c = 0; c < 2 * sc.size(); ++c) {
            const Cand &cd = sc[c < sc.size() ? c : 2 * sc.size() - 1 - c];
            const int d = cd.d, r = cd.r, pl = cd.pl;
            if (st != VIRS_OK) break;
            s->tile_rows = r;
            s->depth = d;
            s->zc = pl;
            s->maps_rows = 0;
            if ((st = ready_to_run(s)) != VIRS_OK) break;
            // one untimed step, then trial_steps timed ones
            cudaError_t e = enqueue_step(s, s->cur, s->stream);
            s->cur ^= 1;
            cudaEventRecord(e0, s->stream);
            for (uint32_t k = 0; k < trial_steps && e == cudaSuccess; ++k) {
                e = enqueue_step(s, s->cur, s->stream);
                s->cur ^= 1;
            }
            cudaEventRecord(e1, s->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) {
                st = cuda_fail(e, "autotune trial");
                break;
            }
            if ((st = check_err(s)) != VIRS_OK) break;
            if (ms / trial_steps < best_ms) {
                best_ms = ms / trial_steps;
                pick.t = {r, pl, d, ms / trial_steps};
            }
            if ((st = reset_state(s)) != VIRS_OK) break;
        }
        // two steps per pass (groups of four steps), with the best single-step
        // tiling for the steps that do not fill a group; not with stochastic
        // rounding, which two steps per pass do not apply
        if (st == VIRS_OK && !sr_on(s)) {
            s->tile_rows = pick.t.tile_rows;
            s->depth = pick.t.pipeline_depth;
            s->zc = pick.t.planes_per_block;
            s->maps_rows = 0;
            // Each candidate is timed twice, in forward and then reverse
            // order: a sustained load brings the GPU to its power cap within
            // about a second, which would favour the candidates timed first.
            std::vector<std::pair<int, int>> cand;
            for (int r : {14, 16, 12})
                for (int pl : {32, 42, 64, 102}) cand.emplace_back(r, pl);
            bool room = true;
            for (size_t c = 0; c < 2 * cand.size() && room; ++c) {
                const int r = cand[c < cand.size() ? c : 2 * cand.size() - 1 - c].first;
                const int pl = cand[c < cand.size() ? c : 2 * cand.size() - 1 - c].second;
                if (st != VIRS_OK) break;
                s->pair_steps = 2;
                s->pair_rows = r;
                s->pair_zc = pl;
                s->pm_rows = 0;
                if ((st = ready_to_run(s)) != VIRS_OK || (st = ready_pairs(s)) != VIRS_OK) break;
                if (!pair_on(s)) { // no room for the spare buffers, or a grid too small
                    room = false;
                    break;
                }
                if ((st = sync_border_planes(s, s->stream)) != VIRS_OK) break;
                cudaError_t e = enqueue_quad(s, s->cur, s->stream);
                cudaEventRecord(e0, s->stream);
                for (uint32_t k = 0; k < quads && e == cudaSuccess; ++k) e = enqueue_quad(s, s->cur, s->stream);
                cudaEventRecord(e1, s->stream);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float ms = 0;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                if (e != cudaSuccess) {
                    st = cuda_fail(e, "autotune trial (two steps per pass)");
                    break;
                }
                if ((st = check_err(s)) != VIRS_OK) break;
                const float per = ms / (4.f * quads);
                if (per < best_ms) {
                    best_ms = per;
                    pick.t.ms_per_step = per;
                    pick.pair_steps = 2;
                    pick.pair_rows = r;
                    pick.pair_zc = pl;
                }
                if ((st = reset_state(s)) != VIRS_OK) break;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st != VIRS_OK) return st;
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune[key] = pick;
    }
    s->tile_rows = pick.t.tile_rows;
    s->zc = pick.t.planes_per_block;
    s->depth = pick.t.pipeline_depth;
    s->maps_rows = 0;
    s->pair_steps = pick.pair_steps;
    s->pair_rows = pick.pair_rows;
    s->pair_zc = pick.pair_zc;
    s->pm_rows = 0;
    if (pick.pair_steps == 1) {
        s->spare[0].release();
        s->spare[1].release();
    }
    s->drop_graphs();
    VIRS_TRY(ready_to_run(s));
    VIRS_TRY(reset_state(s));
    VIRS_CUDA(cudaEventRecord(s->done, s->stream));
    if (best) *best = pick.t;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_get_tiling(const virs_sim *s, virs_tiling *out)
{
    if (!s || !out) return fail(VIRS_E_ARG, "virs_get_tiling: null argument");
    out->tile_rows = s->tile_rows;
    out->planes_per_block = s->zc;
    out->pipeline_depth = s->depth;
    out->ms_per_step = 0.f;
    return VIRS_OK;
}

namespace virs {

// inputs of the allocation-free energy monitor; orders `stream` after the
// handle's queued work with an event (no allocation)
virs_status energy_inputs(virs_sim *s, void *stream, EnergyInputs *in)
{
    if (!s->classified) return fail(VIRS_E_STATE, "grid not classified");
    VIRS_TRY(use_device(s));
    in->p = s->field[s->cur].ptr;
    in->q = s->field[s->cur ^ 1].ptr;
    in->code = s->code.as<uint8_t>();
    in->nx = s->nx;
    in->ny = s->ny;
    in->nz = s->nz;
    in->px = s->px;
    in->storage = s->prm.storage;
    in->device = s->prm.device;
    in->lambda2 = (double)s->c2dt2 * (double)s->inv_h2;
    in->scale2 = (double)s->inv_scale * (double)s->inv_scale;
    in->stream = stream ? (cudaStream_t)stream : s->stream;
    in->done = s->done;
    if (in->stream != s->stream) {
        VIRS_CUDA(cudaEventRecord(s->done, s->stream));
        VIRS_CUDA(cudaStreamWaitEvent(in->stream, s->done, 0));
    }
    return VIRS_OK;
}

} // namespace virs

// ============================================================================
// batched runs: many simulations advanced together, three launches per step
// ============================================================================

struct virs_batch {
    std::vector<virs_sim *> mem;
    std::vector<uint64_t> gen;
    int dev = 0, storage = 0, rows = 8, depth = 2, planes = 0;
    bool persistent = false;
    uint64_t ntiles = 0, nbnd = 0;
    uint32_t max_sections = 0;
    DevBuf desc, err;
    // each member's zero-code masks for the batch's tiling
    std::deque<DevBuf> zmasks;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    static constexpr int GRAPH_STEPS = 32;

    ~virs_batch()
    {
        drop_graphs();
        if (done) cudaEventDestroy(done);
        if (stream) cudaStreamDestroy(stream);
    }
    void drop_graphs()
    {
        for (auto &g : graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }
};

namespace {

virs_status batch_check(const virs_batch *b)
{
    for (size_t i = 0; i < b->mem.size(); ++i) {
        const virs_sim *s = b->mem[i];
        if (s->gen != b->gen[i])
            return fail(VIRS_E_STATE, "batch member " + std::to_string(i) + " changed after the batch was built");
        if (s->cur != b->mem[0]->cur || s->steps_done != b->mem[0]->steps_done)
            return fail(VIRS_E_STATE, "batch members must be at the same step");
    }
    return VIRS_OK;
}

// descriptors of every member for the batch's tiling
virs_status batch_build(virs_batch *b)
{
    b->drop_graphs();
    b->zmasks.clear();
    std::vector<BatchMember> h(b->mem.size());
    uint64_t tiles = 0, bnd = 0;
    b->max_sections = 0;
    const CUtensorMapDataType dt = b->storage == VIRS_STORAGE_F32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : b->storage == VIRS_STORAGE_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                                    : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    for (size_t i = 0; i < b->mem.size(); ++i) {
        virs_sim *s = b->mem[i];
        VIRS_TRY(ready_to_run(s));
        BatchMember &m = h[i];
        std::memset(&m, 0, sizeof(m));
        const size_t el = s->storage_bytes();
        for (int k = 0; k < 2; ++k) {
            VIRS_TRY(encode(&m.mapP[k], dt, el, s->field[k].ptr, s, (uint32_t)tma_box_width(b->storage), b->rows + 2));
            VIRS_TRY(encode(&m.mapQ[k], dt, el, s->field[k].ptr, s, (uint32_t)tma_tile_x(), b->rows));
        }
        VIRS_TRY(encode(&m.mapC, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, s->code.ptr, s, (uint32_t)tma_tile_x(), b->rows));
        const int zc = b->planes > 0 ? b->planes : (s->zc > 0 ? s->zc : default_planes(s->nz));
        const uint64_t *zm = nullptr;
        if (zero_masks_useful(s)) {
            b->zmasks.emplace_back();
            VIRS_TRY(build_zero_masks(s, b->rows, zc, b->zmasks.back()));
            zm = b->zmasks.back().as<uint64_t>();
        }
        for (int par = 0; par < 2; ++par) {
            m.step[par] = step_args(s, par);
            m.step[par].zc = zc;
            m.step[par].stop = nullptr; // batches run every step
            m.step[par].tzmask = zm; // the batch's tiling, not the member's own
            m.post[par] = post_args(s, par);
            m.post[par].stop = nullptr;
        }
        m.bidx = s->bidx.as<uint32_t>();
        m.gx = (s->px + tma_tile_x() - 1) / tma_tile_x();
        m.gy = (s->ny + b->rows - 1) / b->rows;
        m.gz = (s->nz - 2 + zc - 1) / zc;
        m.first_tile = tiles;
        m.first_bnd = bnd;
        tiles += (uint64_t)m.gx * m.gy * m.gz;
        bnd += s->nb;
        b->max_sections = std::max(b->max_sections, s->nsec);
        b->gen[i] = s->gen;
    }
    VIRS_TRY(b->desc.alloc(h.size() * sizeof(BatchMember), "batch descriptors"));
    VIRS_CUDA(copy_on(b->stream, b->desc.ptr, h.data(), h.size() * sizeof(BatchMember), cudaMemcpyHostToDevice));
    b->ntiles = tiles;
    b->nbnd = bnd;
    return VIRS_OK;
}

cudaError_t batch_enqueue(const virs_batch *b, int parity, cudaStream_t st)
{
    const BatchMember *d = b->desc.as<BatchMember>();
    const uint32_t n = (uint32_t)b->mem.size();
    cudaError_t e =
        launch_step_tma_batch(b->storage, b->rows, b->depth, d, n, b->ntiles, parity, b->persistent, b->err.as<int>(), st,
                              sr_on(b->mem[0]));
    if (e != cudaSuccess) return e;
    e = launch_boundary_batch(b->storage, d, n, b->nbnd, parity, b->max_sections, st);
    if (e != cudaSuccess) return e;
    return launch_post_batch(b->storage, d, n, parity, st);
}

virs_status batch_graphs(virs_batch *b, cudaStream_t st)
{
    b->drop_graphs();
    for (int par = 0; par < 2; ++par) {
        cudaGraph_t g = nullptr;
        VIRS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < virs_batch::GRAPH_STEPS && e == cudaSuccess; ++i) e = batch_enqueue(b, par ^ (i & 1), st);
        const cudaError_t e2 = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(e, "capturing the batched step loop");
        }
        if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->graph[par], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    }
    return VIRS_OK;
}

virs_status batch_steps(virs_batch *b, uint64_t n, cudaStream_t st, bool use_graph)
{
    virs_sim *m0 = b->mem[0];
    for (virs_sim *s : b->mem)
        if (s->steps_done + n > s->ircap)
            return fail(VIRS_E_ARG, "a batch member has receiver storage for fewer steps: reserve them with "
                                    "virs_start_simulation");
    for (virs_sim *s : b->mem) {
        VIRS_CUDA(cudaEventRecord(s->done, s->stream));
        VIRS_CUDA(cudaStreamWaitEvent(st, s->done, 0));
    }
    const int cur = m0->cur;
    uint64_t i = 0;
    if (use_graph && n >= (uint64_t)virs_batch::GRAPH_STEPS) {
        if (!b->graph[0]) VIRS_TRY(batch_graphs(b, st));
        for (; i + virs_batch::GRAPH_STEPS <= n; i += virs_batch::GRAPH_STEPS)
            VIRS_CUDA(cudaGraphLaunch(b->graph[cur ^ (int)(i & 1)], st));
    }
    for (; i < n; ++i) {
        const cudaError_t e = batch_enqueue(b, cur ^ (int)(i & 1), st);
        if (e != cudaSuccess) return cuda_fail(e, "batched step launch");
    }
    for (virs_sim *s : b->mem) {
        s->cur ^= (int)(n & 1);
        s->steps_done += n;
        VIRS_CUDA(cudaEventRecord(s->done, st));
    }
    VIRS_CUDA(cudaEventRecord(b->done, st));
    return VIRS_OK;
}

} // namespace

VIRS_EXPORT virs_status virs_batch_create(virs_sim *const *sims, uint32_t n, virs_batch **out)
{
    if (!out || !sims || n == 0) return fail(VIRS_E_ARG, "virs_batch_create: null or empty argument");
    *out = nullptr;
    for (uint32_t i = 0; i < n; ++i) {
        if (!sims[i]) return fail(VIRS_E_ARG, "virs_batch_create: null member");
        if (!started(sims[i])) return fail(VIRS_E_STATE, "batch members must be started (virs_start_simulation)");
        if (sims[i]->prm.device != sims[0]->prm.device || sims[i]->prm.storage != sims[0]->prm.storage)
            return fail(VIRS_E_ARG, "batch members must share the device and the storage type");
        if (sr_on(sims[i]) != sr_on(sims[0]))
            return fail(VIRS_E_ARG, "batch members must share the rounding of their 16-bit stores");
        for (uint32_t j = 0; j < i; ++j)
            if (sims[j] == sims[i]) return fail(VIRS_E_ARG, "a simulation appears twice in the batch");
    }
    std::unique_ptr<virs_batch> b(new (std::nothrow) virs_batch());
    if (!b) return fail(VIRS_E_OOM, "virs_batch_create: host allocation failed");
    b->mem.assign(sims, sims + n);
    b->gen.assign(n, 0);
    b->dev = sims[0]->prm.device;
    b->storage = sims[0]->prm.storage;
    VIRS_TRY(use_device(sims[0]));
    for (virs_sim *s : b->mem) VIRS_TRY(wait_done(s));
    VIRS_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    VIRS_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
    VIRS_TRY(b->err.alloc(sizeof(int), "batch error flag"));
    VIRS_TRY(batch_build(b.get()));
    VIRS_TRY(batch_check(b.get()));
    VIRS_CUDA(cudaEventRecord(b->done, b->stream));
    *out = b.release();
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_batch_destroy(virs_batch *b)
{
    if (!b) return VIRS_OK;
    cudaSetDevice(b->dev);
    cudaStreamSynchronize(b->stream);
    delete b;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_batch_run(virs_batch *b, uint64_t steps, void *stream)
{
    if (!b) return fail(VIRS_E_ARG, "virs_batch_run: null");
    VIRS_CUDA(cudaSetDevice(b->dev));
    VIRS_TRY(batch_check(b));
    if (steps == 0) return VIRS_OK;
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    return batch_steps(b, steps, st, true);
}

VIRS_EXPORT virs_status virs_batch_synchronize(virs_batch *b)
{
    if (!b) return fail(VIRS_E_ARG, "virs_batch_synchronize: null");
    VIRS_CUDA(cudaSetDevice(b->dev));
    VIRS_CUDA(cudaEventSynchronize(b->done));
    int e = 0;
    VIRS_CUDA(copy_on(b->stream, &e, b->err.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        VIRS_CUDA(zero_on(b->stream, b->err.ptr, sizeof(int)));
        return fail(VIRS_E_TIMEOUT, "a batched stencil block gave up waiting for its staged planes");
    }
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_batch_set_tiling(virs_batch *b, int rows, int planes, int depth)
{
    if (!b) return fail(VIRS_E_ARG, "virs_batch_set_tiling: null");
    if (rows != 0 && rows != 4 && rows != 8 && rows != 16) return fail(VIRS_E_ARG, "tile rows must be 4, 8 or 16");
    if (planes < 0 || planes > 4096) return fail(VIRS_E_ARG, "planes per block must be 0..4096");
    if (depth < -1 || depth == 0 || depth > 3) return fail(VIRS_E_ARG, "batched runs use the TMA kernel: depth -1 or 1..3");
    VIRS_CUDA(cudaSetDevice(b->dev));
    VIRS_CUDA(cudaEventSynchronize(b->done));
    b->rows = rows ? rows : 8;
    b->planes = planes;
    b->depth = depth < 0 ? 2 : depth;
    return batch_build(b);
}

VIRS_EXPORT virs_status virs_batch_autotune(virs_batch *b, uint32_t trial_steps, virs_tiling *best)
{
    if (!b) return fail(VIRS_E_ARG, "virs_batch_autotune: null");
    if (trial_steps == 0 || trial_steps > 1000) return fail(VIRS_E_ARG, "trial_steps must be 1..1000");
    VIRS_CUDA(cudaSetDevice(b->dev));
    VIRS_TRY(batch_check(b));
    for (virs_sim *s : b->mem) {
        if (s->steps_done != 0) return fail(VIRS_E_STATE, "virs_batch_autotune must run before the first step");
        if (s->ircap < 2ull * trial_steps + 2) return fail(VIRS_E_ARG, "reserve at least 2*trial_steps+2 steps");
    }
    cudaEvent_t e0, e1;
    VIRS_CUDA(cudaEventCreate(&e0));
    VIRS_CUDA(cudaEventCreate(&e1));
    virs_tiling pick{8, 0, 2, 0.f};
    bool pick_persistent = false;
    float best_ms = 1e30f;
    virs_status st = VIRS_OK;
    // every candidate timed twice, in forward and then reverse order (the
    // power cap would favour the candidates timed first)
    struct Cand {
        int pers, d, r, pl;
    };
    std::vector<Cand> cand;
    for (int pers : {0, 1})
        for (int d : {1, 2, 3})
            for (int r : {4, 8, 16})
                for (int pl : {8, 16, 32, 64}) cand.push_back({pers, d, r, pl});
    for (size_t c = 0; c < 2 * cand.size(); ++c) {
        const Cand &cd = cand[c < cand.size() ? c : 2 * cand.size() - 1 - c];
        const int pers = cd.pers, d = cd.d, r = cd.r, pl = cd.pl;
        if (st != VIRS_OK) break;
        b->rows = r;
        b->depth = d;
        b->planes = pl;
        b->persistent = pers != 0;
        if ((st = batch_build(b)) != VIRS_OK) break;
        if ((st = batch_steps(b, 1, b->stream, false)) != VIRS_OK) break;
        cudaEventRecord(e0, b->stream);
        if ((st = batch_steps(b, trial_steps, b->stream, false)) != VIRS_OK) break;
        cudaEventRecord(e1, b->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "batch autotune trial");
            break;
        }
        if (ms < best_ms) {
            best_ms = ms;
            pick = {r, pl, d, ms / trial_steps};
            pick_persistent = pers != 0;
        }
        for (virs_sim *s : b->mem)
            if ((st = reset_state(s)) != VIRS_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != VIRS_OK) return st;
    b->rows = pick.tile_rows;
    b->depth = pick.pipeline_depth;
    b->planes = pick.planes_per_block;
    b->persistent = pick_persistent;
    VIRS_TRY(batch_build(b));
    VIRS_TRY(virs_batch_synchronize(b));
    if (best) *best = pick;
    return VIRS_OK;
}

// ============================================================================
// adjoint
// ============================================================================

VIRS_EXPORT virs_status virs_forward_checkpointed(virs_sim *s, uint64_t steps, uint32_t every, void *stream)
{
    if (!s) return fail(VIRS_E_ARG, "virs_forward_checkpointed: null");
    if (steps == 0 || every == 0 || every > 4096) return fail(VIRS_E_ARG, "need steps > 0 and 1 <= every <= 4096");
    if (s->prm.storage != VIRS_STORAGE_F32) return fail(VIRS_E_ARG, "the adjoint runs with FP32 storage");
    if (s->depth == 0) return fail(VIRS_E_STATE, "the adjoint needs the TMA kernel (pipeline depth 1..3)");
    if (s->prm.rigid_walls)
        return fail(VIRS_E_STATE, "the adjoint assumes the mirrored update at boundary voxels, not rigid_walls");
    if (s->stop_rule) return fail(VIRS_E_STATE, "the adjoint runs every step: disable the stop rule (virs_set_stop_rule)");
    VIRS_TRY(virs_start_simulation(s, steps));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    auto &A = s->adj;
    A.ready = false;
    A.steps = steps;
    A.every = every;
    A.nck = (steps + every - 1) / every;
    const size_t fb = s->nvox * 4, sb = state_bytes(s);
    VIRS_TRY(A.ckp.alloc(A.nck * fb, "checkpoints"));
    VIRS_TRY(A.ckq.alloc(A.nck * fb, "checkpoints"));
    VIRS_TRY(A.cks.alloc(A.nck * sb, "checkpoints"));
    VIRS_CUDA(cudaEventRecord(s->done, s->stream));
    VIRS_CUDA(cudaStreamWaitEvent(st, s->done, 0));
    for (uint64_t c = 0; c < A.nck; ++c) {
        VIRS_CUDA(cudaMemcpyAsync(A.ckp.as<char>() + c * fb, s->field[s->cur].ptr, fb, cudaMemcpyDeviceToDevice, st));
        VIRS_CUDA(cudaMemcpyAsync(A.ckq.as<char>() + c * fb, s->field[s->cur ^ 1].ptr, fb, cudaMemcpyDeviceToDevice, st));
        VIRS_CUDA(cudaMemcpyAsync(A.cks.as<char>() + c * sb, s->state.ptr, sb, cudaMemcpyDeviceToDevice, st));
        VIRS_TRY(run_steps(s, std::min<uint64_t>(every, steps - c * every), st));
    }
    A.gen = s->gen;
    A.ready = true;
    return VIRS_OK;
}

VIRS_EXPORT virs_status virs_adjoint(virs_sim *s, const float *dl_dir, double *grad_coef, float *grad_signal)
{
    if (!s || !dl_dir) return fail(VIRS_E_ARG, "virs_adjoint: null argument");
    auto &A = s->adj;
    if (!A.ready || A.gen != s->gen || s->steps_done != A.steps || !s->fields_valid)
        return fail(VIRS_E_STATE, "call virs_forward_checkpointed first (and change nothing in between)");
    VIRS_TRY(use_device(s));
    VIRS_TRY(wait_done(s));
    cudaStream_t st = s->stream;
    const uint64_t steps = A.steps, every = A.every, nb = s->nb;
    // forward states (shared cascade layout) and the adjoint's own state
    // adjoints, four per section
    const size_t fb = s->nvox * 4, sb = state_bytes(s), sba = std::max<uint64_t>(nb, 1) * s->nsec * 4 * 4;
    const uint32_t ncoef = s->nmat * s->nsec * 5;
    VIRS_TRY(A.segrec.alloc(every * std::max<uint64_t>(nb, 1) * sizeof(float4), "adjoint segment records"));
    VIRS_TRY(A.segst.alloc(every * sb, "adjoint segment states"));
    for (int k = 0; k < 2; ++k) VIRS_TRY(A.buf[k].alloc(fb, "adjoint field"));
    VIRS_TRY(A.ast.alloc(sba, "adjoint filter states"));
    VIRS_TRY(A.dbar.alloc(std::max<uint64_t>(nb, 1) * 4, "adjoint boundary terms"));
    VIRS_TRY(A.cq.alloc(std::max<uint64_t>(nb, 1) * 4, "adjoint boundary terms"));
    VIRS_TRY(A.grad.alloc(ncoef * sizeof(double), "coefficient gradients"));
    VIRS_TRY(A.dl.alloc(std::max<uint32_t>(s->nrcv, 1) * steps * 4, "loss gradient"));
    VIRS_TRY(A.gsig.alloc(std::max<uint32_t>(s->nsrc, 1) * steps * 4, "signal gradients"));
    if (s->nrcv) VIRS_CUDA(copy_on(s->stream, A.dl.ptr, dl_dir, (size_t)s->nrcv * steps * 4, cudaMemcpyHostToDevice));
    const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    for (int k = 0; k < 2; ++k) {
        VIRS_TRY(encode(&A.mapP[k], dt, 4, A.buf[k].ptr, s, (uint32_t)tma_box_width(VIRS_STORAGE_F32), s->tile_rows + 2));
        VIRS_TRY(encode(&A.mapQ[k], dt, 4, A.buf[k].ptr, s, (uint32_t)tma_tile_x(), s->tile_rows));
    }
    VIRS_TRY(ready_to_run(s));
    int t = 0; // A.buf[t] holds T, A.buf[t ^ 1] holds RR
    for (int64_t c = (int64_t)A.nck - 1; c >= 0; --c) {
        const uint64_t n0 = (uint64_t)c * every, n1 = std::min<uint64_t>(n0 + every, steps);
        // rebuild the segment: restore the checkpoint and run forward, keeping
        // the states before every step and the stencil's boundary records
        s->cur = 0;
        VIRS_CUDA(cudaMemcpyAsync(s->field[0].ptr, A.ckp.as<char>() + c * fb, fb, cudaMemcpyDeviceToDevice, st));
        VIRS_CUDA(cudaMemcpyAsync(s->field[1].ptr, A.ckq.as<char>() + c * fb, fb, cudaMemcpyDeviceToDevice, st));
        VIRS_CUDA(cudaMemcpyAsync(A.segst.ptr, A.cks.as<char>() + c * sb, sb, cudaMemcpyDeviceToDevice, st));
        VIRS_CUDA(launch_set_u32(s->ctr.as<uint32_t>(), (uint32_t)n0, st));
        for (uint64_t n = n0; n < n1; ++n) {
            const uint64_t k = n - n0;
            cudaError_t e = launch_stencil(s, s->cur, st);
            // the boundary pass keeps its records straight in the segment's
            // slot k, and reads the states before the step from slot k and
            // writes those after it to slot k + 1 (the last step's to the
            // handle's own states)
            StepArgs ka = step_args(s, s->cur);
            ka.side = A.segrec.as<float4>() + k * nb;
            ka.state = reinterpret_cast<float *>(A.segst.as<char>() + k * sb);
            ka.state_out = k + 1 < every ? reinterpret_cast<float *>(A.segst.as<char>() + (k + 1) * sb)
                                         : s->state.as<float>();
            if (e == cudaSuccess) e = launch_boundary(s->prm.storage, ka, BND_KEEP, st);
            if (e == cudaSuccess) e = launch_post(s->prm.storage, post_args(s, s->cur), st);
            if (e != cudaSuccess) return cuda_fail(e, "adjoint recomputation");
            s->cur ^= 1;
        }
        // reverse steps of the segment
        for (int64_t n = (int64_t)n1 - 1; n >= (int64_t)n0; --n) {
            const uint64_t k = (uint64_t)n - n0;
            float *T = A.buf[t].as<float>(), *RR = A.buf[t ^ 1].as<float>();
            cudaError_t e = launch_adj_inject(T, s->code.as<uint8_t>(), s->rcv.as<uint64_t>(), s->nrcv, A.dl.as<float>(),
                                              steps, (uint64_t)n, s->src.as<uint64_t>(), s->nsrc, A.gsig.as<float>(),
                                              steps, st);
            if (e == cudaSuccess)
                e = launch_adj_boundary(T, s->bidx.as<uint32_t>(), s->bmat.as<uint8_t>(), s->bw.as<float>(),
                                        s->coef.as<float>(), A.segrec.as<float4>() + k * nb,
                                        reinterpret_cast<const float *>(A.segst.as<char>() + k * sb), A.ast.as<float>(),
                                        A.dbar.as<float>(), A.cq.as<float>(), A.grad.as<double>(), nb, s->nx, s->ny,
                                        s->px, s->nsec, s->nmat, s->prm.boundary_form, (double)s->K,
                                        s->prm.mix_filtered, s->prm.mix_direct, (double)s->prm.boundary_gain, st);
            if (e == cudaSuccess) {
                StepArgs a = step_args(s, 0);
                a.p = T;
                a.q = RR;
                a.nhard = 0;
                const TmaMaps m{&A.mapP[t], &A.mapQ[t ^ 1], &s->tmC};
                e = launch_step_tma(VIRS_STORAGE_F32, s->tile_rows, s->depth, a, m, s->err.as<int>(), st);
                if (e == cudaSuccess) e = launch_zero_at(RR, s->hpos.as<uint32_t>(), s->nhpos, st);
                // the free value A F - RR at the boundary voxels, which the
                // stencil left alone
                if (e == cudaSuccess) e = launch_boundary(VIRS_STORAGE_F32, a, BND_RECORD, st);
            }
            if (e == cudaSuccess)
                e = launch_adj_fix(RR, T, s->bidx.as<uint32_t>(), s->side.as<float4>(), A.dbar.as<float>(),
                                   A.cq.as<float>(), nb, s->nx, s->ny, s->px, st);
            if (e != cudaSuccess) return cuda_fail(e, "adjoint step");
            t ^= 1;
        }
    }
    VIRS_CUDA(cudaStreamSynchronize(st));
    VIRS_TRY(check_err(s));
    if (grad_coef) VIRS_CUDA(copy_on(s->stream, grad_coef, A.grad.ptr, ncoef * sizeof(double), cudaMemcpyDeviceToHost));
    if (grad_signal && s->nsrc)
        VIRS_CUDA(copy_on(s->stream, grad_signal, A.gsig.ptr, (size_t)s->nsrc * steps * 4, cudaMemcpyDeviceToHost));
    // the fields now hold an intermediate forward state
    s->fields_valid = false;
    VIRS_CUDA(cudaEventRecord(s->done, st));
    return VIRS_OK;
}
