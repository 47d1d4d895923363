// device.cu -- uploads of the packed matrix and its tilings.
#include "device.hpp"

#include <cstdlib>
#include <mutex>
#include <string>

namespace pdfp {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

namespace {
constexpr int kMaxPoolDevices = 64;
constexpr uint64_t kPoolKeepBytes = 256ull << 20;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};
bool g_pool_failed[kMaxPoolDevices] = {};
int g_pool_enabled = -1;  // -1: not read yet

cudaMemPool_t current_pool() {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (g_pool_enabled < 0) {
        const char* e = std::getenv("PDFP_POOL");
        g_pool_enabled = (e && e[0] == '0') ? 0 : 1;
    }
    if (!g_pool_enabled) return nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxPoolDevices) return nullptr;
    if (g_pools[dev] || g_pool_failed[dev]) return g_pools[dev];
    int supported = 0;
    cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev);
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (!supported || cudaMemPoolCreate(&g_pools[dev], &props) != cudaSuccess) {
        g_pools[dev] = nullptr;
        g_pool_failed[dev] = true;
        cudaGetLastError();
        return nullptr;
    }
    uint64_t keep = kPoolKeepBytes;
    cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    return g_pools[dev];
}
}  // namespace

namespace {
constexpr int kPinnedClasses = 32;
constexpr size_t kPinnedKeep = 8;  // blocks kept per size class
std::mutex g_pinned_mu;
std::vector<void*> g_pinned_free[kPinnedClasses];
int pinned_class(size_t bytes) {
    int c = 0;
    while ((size_t(256) << c) < bytes && c < kPinnedClasses - 1) ++c;
    return c;
}
}  // namespace

void* pinned_take(size_t bytes) {
    const int c = pinned_class(bytes);
    if ((size_t(256) << c) < bytes) throw Error(E_INVALID, "pinned block too large");
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        if (!g_pinned_free[c].empty()) {
            void* p = g_pinned_free[c].back();
            g_pinned_free[c].pop_back();
            return p;
        }
    }
    void* p = nullptr;
    PDFP_CK(cudaMallocHost(&p, size_t(256) << c));
    return p;
}

void pinned_give(void* p, size_t bytes) {
    if (!p) return;
    const int c = pinned_class(bytes);
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        if (g_pinned_free[c].size() < kPinnedKeep) {
            g_pinned_free[c].push_back(p);
            return;
        }
    }
    cudaFreeHost(p);
}

void* arena_malloc(size_t bytes, bool* pooled) {
    void* p = nullptr;
    *pooled = false;
    if (cudaMemPool_t pool = current_pool()) {
        // on the legacy default stream, then waited for: the memory is zero and
        // usable from every stream when this returns
        PDFP_CK(cudaMallocFromPoolAsync(&p, bytes, pool, 0));
        *pooled = true;
        cudaError_t e = cudaMemsetAsync(p, 0, bytes, 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
        if (e != cudaSuccess) {
            cudaFreeAsync(p, 0);
            throw Error(E_CUDA, std::string("arena zero-fill: ") + cudaGetErrorString(e));
        }
        return p;
    }
    PDFP_CK(cudaMalloc(&p, bytes));
    cudaError_t e = cudaMemset(p, 0, bytes);
    if (e != cudaSuccess) {
        cudaFree(p);
        throw Error(E_CUDA, std::string("arena zero-fill: ") + cudaGetErrorString(e));
    }
    return p;
}

void arena_free(const std::vector<void*>& ptrs, const std::vector<bool>& pooled) {
    // no kernel of any stream may still use the memory (cudaFree's own guarantee)
    cudaDeviceSynchronize();
    for (size_t i = 0; i < ptrs.size(); ++i) {
        if (pooled[i]) cudaFreeAsync(ptrs[i], 0); else cudaFree(ptrs[i]);
    }
    cudaStreamSynchronize(0);
}
const char* last_error_cstr() { return g_last_error.c_str(); }

__global__ void f64_to_f32_kernel(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        b[i] = static_cast<float>(a[i]);
}

template <class T>
static std::pair<const void*, size_t> part(const std::vector<T>& v) {
    return {v.data(), v.size() * sizeof(T)};
}

void DeviceMatrix::upload(DeviceArena& ar, bool want_f32) {
    const std::vector<void*> d = ar.upload_group(
        {part(L.A.rp), part(L.A.ci), part(L.A.v), part(L.At.rp), part(L.At.ci), part(L.At.v),
         part(L.row_off), part(L.col_off), part(L.n_eq), part(L.row_orig), part(L.col_orig)});
    rp_a = static_cast<int32_t*>(d[0]);
    ci_a = static_cast<int32_t*>(d[1]);
    v64_a = static_cast<double*>(d[2]);
    rp_t = static_cast<int32_t*>(d[3]);
    ci_t = static_cast<int32_t*>(d[4]);
    v64_t = static_cast<double*>(d[5]);
    row_off = static_cast<int32_t*>(d[6]);
    col_off = static_cast<int32_t*>(d[7]);
    n_eq = static_cast<int32_t*>(d[8]);
    row_orig = static_cast<int32_t*>(d[9]);
    col_orig = static_cast<int32_t*>(d[10]);
    max_m = max_n = 0;
    for (int p = 0; p < L.K; ++p) {
        max_m = std::max(max_m, L.row_off[p + 1] - L.row_off[p]);
        max_n = std::max(max_n, L.col_off[p + 1] - L.col_off[p]);
    }
    if (want_f32) {
        v32_a = ar.alloc<float>(L.NNZ);
        v32_t = ar.alloc<float>(L.NNZ);
        refresh_f32(0);
        PDFP_CK(cudaDeviceSynchronize());
    }
}

__global__ void recip_kernel(const double* __restrict__ s, double* __restrict__ d, int64_t n) {
    for (int64_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += int64_t(gridDim.x) * 256)
        d[i] = __ddiv_rn(1.0, s[i]);
}

void cast_f64_to_f32(const double* src, float* dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4096));
    f64_to_f32_kernel<<<blocks, 256, 0, s>>>(src, dst, n);
    PDFP_CK(cudaGetLastError());
}

void reciprocal(const double* src, double* dst, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4096));
    recip_kernel<<<blocks, 256, 0, s>>>(src, dst, n);
    PDFP_CK(cudaGetLastError());
}

void DeviceMatrix::refresh_f32(cudaStream_t s) {
    if (!v32_a || L.NNZ == 0) return;
    int blocks = static_cast<int>(std::min<int64_t>((L.NNZ + 255) / 256, 4096));
    f64_to_f32_kernel<<<blocks, 256, 0, s>>>(v64_a, v32_a, L.NNZ);
    f64_to_f32_kernel<<<blocks, 256, 0, s>>>(v64_t, v32_t, L.NNZ);
    PDFP_CK(cudaGetLastError());
}

// Upload a built tiling of the CSR whose device arrays are rp / ci.
static DeviceMatrix::Tiling upload_tiling(DeviceArena& ar, DeviceMatrix::Tiling&& t, int32_t rows,
                                          const int32_t* rp, const int32_t* ci, const StageGeom& g) {
    SideDev& s = t.dev;
    s.rows = rows;
    s.n_tiles = static_cast<int32_t>(t.host.tile_inst.size());
    s.n_chunks = static_cast<int32_t>(t.host.chunk_k0.size());
    s.max_tile_rows = t.host.max_tile_rows;
    s.stage_bytes = g.stage_bytes;
    s.rp = rp;
    s.ci = ci;
    std::vector<ChunkDesc> desc(t.host.chunk_k0.size());
    for (size_t c = 0; c < desc.size(); ++c) {
        const int32_t tile = t.host.chunk_tile[c];
        desc[c] = ChunkDesc{t.host.chunk_k0[c], t.host.chunk_k1[c], t.host.tile_row[tile],
                            t.host.tile_row_end[tile], tile, t.host.tile_inst[tile],
                            t.host.chunk_flags[c], t.host.tile_chunk[tile] == (int32_t)c ? 1 : 0};
    }
    const std::vector<void*> d = ar.upload_group({part(t.host.tile_row), part(t.host.tile_chunk),
                                                  part(t.host.tile_inst), part(desc),
                                                  part(t.host.inst_tile0)});
    s.tile_row = static_cast<const int32_t*>(d[0]);
    s.tile_chunk = static_cast<const int32_t*>(d[1]);
    s.tile_inst = static_cast<const int32_t*>(d[2]);
    s.chunks = static_cast<const ChunkDesc*>(d[3]);
    t.inst_tile0 = static_cast<int32_t*>(d[4]);
    return std::move(t);
}

DeviceMatrix::Tiling DeviceMatrix::make_tiling(DeviceArena& ar, bool transpose,
                                               const StageGeom& g,
                                               const std::vector<uint8_t>* skip) const {
    Tiling t;
    const HostCsr& csr = transpose ? L.At : L.A;
    build_tiling(csr, transpose ? L.col_off : L.row_off, g, t.host, skip);
    return upload_tiling(ar, std::move(t), csr.rows, transpose ? rp_t : rp_a, transpose ? ci_t : ci_a, g);
}

bool DeviceMatrix::make_seg(DeviceArena& ar, int nseg, int long_min, const StageGeom& g,
                            SegDev& d, Tiling& pairs, std::vector<uint8_t>& is_long) const {
    HostSeg h;
    if (!build_seg(L.A, L.row_off, nseg, long_min, h)) return false;
    const int64_t nl = static_cast<int64_t>(h.long_row.size());
    d = SegDev();
    d.nseg = h.nseg;
    d.seg_len = h.seg_len;
    d.n_cols = h.n_cols;
    d.n_long = static_cast<int32_t>(nl);
    d.long_row = ar.upload(h.long_row);
    d.long_inst = ar.upload(h.long_inst);
    std::vector<float> v32(h.pairs.v.size());
    for (size_t k = 0; k < v32.size(); ++k) v32[k] = static_cast<float>(h.pairs.v[k]);  // as refresh_f32 rounds
    d.val = ar.upload(v32);
    d.partial = ar.alloc<float>(static_cast<size_t>(nl) * nseg);
    // tiles of the pairs, the segments as instances, interleaved one block per segment
    std::vector<int32_t> off(nseg + 1);
    for (int s = 0; s <= nseg; ++s) off[s] = static_cast<int32_t>(s * nl);
    HostTiling by_seg;
    build_tiling(h.pairs, off, g, by_seg);
    Tiling t;
    interleave_tiles(by_seg, nseg, t.host);
    const int32_t* rp = ar.upload(h.pairs.rp);
    const int32_t* ci = ar.upload(h.pairs.ci);
    pairs = upload_tiling(ar, std::move(t), h.pairs.rows, rp, ci, g);
    is_long.swap(h.is_long);
    return true;
}

VecDev DeviceMatrix::make_vec(DeviceArena& ar, bool transpose, int lane_nnz, int64_t min_items) const {
    const HostCsr& csr = transpose ? L.At : L.A;
    const std::vector<int32_t>& off = transpose ? L.col_off : L.row_off;
    std::vector<VecItem> items;
    int32_t slots = 0;
    if (min_items > 0) {
        // four times the default rows per item (fewer items to fetch per warp) while
        // that still leaves at least min_items items for the warps of the grid
        slots = build_vec_items(csr, off, lane_nnz, items, std::max(1, 32 / std::max(1, lane_nnz)));
        if (static_cast<int64_t>(items.size()) < min_items) items.clear();
    }
    if (items.empty()) slots = build_vec_items(csr, off, lane_nnz, items);
    VecDev v;
    v.n_items = static_cast<int32_t>(items.size());
    v.n_slots = slots;
    v.rp = transpose ? rp_t : rp_a;
    v.ci = transpose ? ci_t : ci_a;
    v.items = ar.upload(items);
    v.piece_sum = ar.alloc<double>(slots > 0 ? slots : 1);  // zero-filled
    v.piece_cnt = ar.alloc<int32_t>(slots > 0 ? slots : 1);
    return v;
}

}  // namespace pdfp
