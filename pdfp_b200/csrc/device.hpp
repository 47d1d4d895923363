// device.hpp -- device memory ownership, errors, and the uploaded matrix.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "layout.hpp"

namespace pdfp {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Status codes (mirror include/pdfp_b200.h).
enum : int { E_INVALID = -1, E_CUDA = -2, E_NOMEM = -3, E_TIMEOUT = -4, E_UNSUPPORTED = -5,
             E_NODEVICE = -6 };

void set_last_error(const std::string& msg);

#define PDFP_CK(expr)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            throw ::pdfp::Error(e_ == cudaErrorMemoryAllocation ? ::pdfp::E_NOMEM                \
                                                                : ::pdfp::E_CUDA,               \
                                std::string(#expr) + ": " + cudaGetErrorString(e_));            \
        }                                                                                       \
    } while (0)

// Device memory behind the arenas.  By default it comes from a library-owned,
// stream-ordered memory pool per device that keeps up to 256 MB of freed memory
// for reuse, so that the many small handles of a pump run (scaling, root LP,
// projector, power iteration) do not pay a driver allocation and a device-wide
// free for each of their buffers; PDFP_POOL=0, or a device without memory pools,
// uses cudaMalloc / cudaFree.  arena_malloc returns zero-filled memory that any
// stream may use; arena_free waits for the whole device first (as cudaFree does).
void* arena_malloc(size_t bytes, bool* pooled);
void arena_free(const std::vector<void*>& ptrs, const std::vector<bool>& pooled);

// Page-locked host blocks for the handles' small poll buffers, kept for reuse by size
// class (powers of two from 256 bytes): pinning host memory costs tens of
// microseconds and unpinning it waits for the device, which a pump run's short-lived
// handles would otherwise pay each time.  The blocks are not zeroed.
void* pinned_take(size_t bytes);
void pinned_give(void* p, size_t bytes);

// Owns device allocations; every buffer is zero-filled, starts 256-byte aligned and
// is padded by 64 bytes so that 16-byte-rounded bulk copies of any sub-range stay
// inside it.  Buffers up to kSmallBytes are carved out of kSlabBytes slabs, each
// zero-filled once: a small handle's dozens of buffers then cost a couple of
// allocations and host waits instead of one each.
class DeviceArena {
  public:
    static constexpr size_t kSlabBytes = size_t(1) << 20;
    static constexpr size_t kSmallBytes = size_t(128) << 10;
    DeviceArena() = default;
    DeviceArena(const DeviceArena&) = delete;
    DeviceArena& operator=(const DeviceArena&) = delete;
    ~DeviceArena() { release(); }
    template <class T>
    T* alloc(size_t n) {
        const size_t bytes = ((n * sizeof(T) + 63) & ~size_t(63)) + 64;
        bytes_ += bytes;
        if (bytes <= kSmallBytes) {
            const size_t off = (slab_used_ + 255) & ~size_t(255);
            if (!slab_ || off + bytes > kSlabBytes) {
                slab_ = static_cast<unsigned char*>(take(kSlabBytes));
                slab_used_ = 0;
                return carve<T>(0, bytes);
            }
            return carve<T>(off, bytes);
        }
        return static_cast<T*>(take(bytes));
    }
    template <class T>
    T* upload(const std::vector<T>& h) {
        T* d = alloc<T>(h.size());
        if (!h.empty()) PDFP_CK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
        return d;
    }
    // Several host arrays {pointer, bytes} uploaded with one copy when together they
    // take at most kGroupBytes: each gets its own 256-byte aligned, 64-byte padded,
    // zero-filled region of one allocation (the layout alloc() gives separate
    // buffers); larger groups go one array at a time.  A small handle's dozens of
    // arrays then cost one host-to-device copy instead of one each.
    static constexpr size_t kGroupBytes = size_t(8) << 20;
    std::vector<void*> upload_group(const std::vector<std::pair<const void*, size_t>>& parts) {
        std::vector<void*> out(parts.size(), nullptr);
        std::vector<size_t> off(parts.size());
        size_t total = 0;
        for (size_t i = 0; i < parts.size(); ++i) {
            off[i] = total;
            total = (total + parts[i].second + 64 + 255) & ~size_t(255);
        }
        if (total > kGroupBytes) {
            for (size_t i = 0; i < parts.size(); ++i) {
                unsigned char* d = alloc<unsigned char>(parts[i].second);
                if (parts[i].second)
                    PDFP_CK(cudaMemcpy(d, parts[i].first, parts[i].second, cudaMemcpyHostToDevice));
                out[i] = d;
            }
            return out;
        }
        unsigned char* d = alloc<unsigned char>(total);
        std::vector<unsigned char> h(total, 0);
        for (size_t i = 0; i < parts.size(); ++i) {
            if (parts[i].second) std::memcpy(h.data() + off[i], parts[i].first, parts[i].second);
            out[i] = d + off[i];
        }
        if (total) PDFP_CK(cudaMemcpy(d, h.data(), total, cudaMemcpyHostToDevice));
        return out;
    }
    void release() {
        if (!ptrs_.empty()) arena_free(ptrs_, pooled_);
        ptrs_.clear();
        pooled_.clear();
        bytes_ = 0;
        slab_ = nullptr;
        slab_used_ = 0;
    }
    size_t bytes() const { return bytes_; }

  private:
    void* take(size_t bytes) {
        bool pooled = false;
        void* p = arena_malloc(bytes, &pooled);
        ptrs_.push_back(p);
        pooled_.push_back(pooled);
        return p;
    }
    template <class T>
    T* carve(size_t off, size_t bytes) {
        slab_used_ = off + bytes;
        return reinterpret_cast<T*>(slab_ + off);
    }
    unsigned char* slab_ = nullptr;  // the slab small buffers are carved from
    size_t slab_used_ = 0;
    std::vector<void*> ptrs_;
    std::vector<bool> pooled_;
    size_t bytes_ = 0;
};

// The packed matrix of a batch on the device: A and A' in FP64 (+FP32 copies
// when asked), index maps, and any number of tilings.
class DeviceMatrix {
  public:
    HostLayout L;
    int32_t *rp_a = nullptr, *ci_a = nullptr, *rp_t = nullptr, *ci_t = nullptr;
    double *v64_a = nullptr, *v64_t = nullptr;
    float *v32_a = nullptr, *v32_t = nullptr;
    int32_t *row_off = nullptr, *col_off = nullptr, *n_eq = nullptr;
    int32_t *row_orig = nullptr, *col_orig = nullptr;
    int32_t max_m = 0, max_n = 0;

    // Upload L (which must already be built) and, if want_f32, FP32 values.
    void upload(DeviceArena& ar, bool want_f32);
    // Refresh the FP32 copies from the FP64 values (after scaling on device).
    void refresh_f32(cudaStream_t s);

    struct Tiling {
        HostTiling host;
        SideDev dev{};
        int32_t* inst_tile0 = nullptr;  // device copy, K + 1
    };
    // Build and upload a tiling of A (transpose = false) or A', leaving out the
    // rows `skip` marks (build_tiling).
    Tiling make_tiling(DeviceArena& ar, bool transpose, const StageGeom& g,
                       const std::vector<uint8_t>* skip = nullptr) const;
    // Build and upload the vec engine's items of A (transpose = false) or A'
    // (build_vec_items), with zeroed piece slots and counters; items of four times the
    // default rows when min_items > 0 and that still gives at least min_items items.
    VecDev make_vec(DeviceArena& ar, bool transpose, int lane_nnz, int64_t min_items) const;
    // Build and upload A's long rows by column segment (build_seg) and a tiling of
    // their (segment, long row) pairs in stage geometry g, interleaved one block per
    // segment (interleave_tiles); false when no row qualifies.  `is_long` receives
    // the rows it took (for the tiling of the rest).
    bool make_seg(DeviceArena& ar, int nseg, int long_min, const StageGeom& g, SegDev& out,
                  Tiling& pairs, std::vector<uint8_t>& is_long) const;
};

// dst[i] = src[i] rounded to FP32, and dst[i] = 1 / src[i] (correctly rounded), on a stream.
void cast_f64_to_f32(const double* src, float* dst, int64_t n, cudaStream_t s);
void reciprocal(const double* src, double* dst, int64_t n, cudaStream_t s);

// scale_problem's arithmetic (src/preconditioner.jl:26-99: Ruiz rounds, Pock-Chambolle
// with alpha, optionally the bound/objective rescaling) applied in place to an uploaded
// matrix in the caller's order (both sides), and to the device vectors vin = {c, lb,
// ub, con_lb, con_ub}, written scaled to vout; D_r, D_c and scales = {bound scale,
// objective scale} (1 without rescaling) to device memory.  Stream-ordered, no host
// synchronisation (precond.cu).
void scale_uploaded(const DeviceMatrix& M, DeviceArena& ar, int32_t ruiz_iterations, double alpha,
                    bool rescale, const double* const vin[5], double* const vout[5], double* D_r,
                    double* D_c, double* scales, cudaStream_t st);

}  // namespace pdfp
