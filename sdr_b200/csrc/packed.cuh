// Packed launches: one launch per substep operation for many scenes.
//
// A solver's phase methods issue every kernel, memset and copy of a substep
// through Solver::issue / mset / mcopy. Normally these launch at once on the
// solver's stream. While a Packer is attached they are recorded instead: per
// scene, the operation's kernel body, its block count and its arguments. Once
// every scene of a batch has recorded its substep, the Packer lines up the
// scenes' operations (each call site, and each repetition of it within the
// substep, is one slot, in the order the code issues them) and launches every
// slot once for all scenes: a ragged offset table gives each scene its range
// of virtual blocks, and the launch's CTAs walk the virtual blocks (a
// persistent grid when there are more of them than the grid holds), each
// running the kernel body with that scene's arguments and its block index
// within the scene. The scenes run exactly the code and arguments they run
// alone, so their results are the same bit for bit.
#pragma once
#include <cuda/std/tuple>
#include <cuda/std/utility>

#include <cstring>
#include <map>
#include <vector>

#include "common.cuh"

namespace sdr {

// Header of one slot's table in the device arena.
struct PackHdr {
    uint32_t ns;       // scenes in this slot
    uint32_t total;    // virtual blocks over all of them
    uint32_t off_at;   // byte offset (from the header) of the ns + 1 block offsets
    uint32_t args_at;  // byte offset of the argument tuples
    uint32_t stride;   // bytes per argument tuple
    uint32_t pad[3];
};

template <class Op, class Tup, size_t... I>
__device__ __forceinline__ void pack_call(VB vb, const Tup& t, cuda::std::index_sequence<I...>) {
    Op::run(vb, cuda::std::get<I>(t)...);
}

// One slot of a packed substep: CTAs take virtual blocks in turn; each finds
// its scene in the offset table (binary search) and runs the body with that
// scene's arguments.
template <class Op, class Tup>
__global__ void __launch_bounds__(Op::kThreads, 1) k_packed(const unsigned char* __restrict__ hdr_p) {
    const PackHdr h = *reinterpret_cast<const PackHdr*>(hdr_p);
    const uint32_t* off = reinterpret_cast<const uint32_t*>(hdr_p + h.off_at);
    for (uint32_t v = blockIdx.x; v < h.total; v += gridDim.x) {
        uint32_t lo = 0, hi = h.ns;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (off[mid] <= v) lo = mid;
            else hi = mid;
        }
        const Tup& t = *reinterpret_cast<const Tup*>(hdr_p + h.args_at + (size_t)lo * h.stride);
        pack_call<Op>(VB{v - off[lo], off[lo + 1] - off[lo]}, t,
                      cuda::std::make_index_sequence<cuda::std::tuple_size<Tup>::value>{});
        __syncthreads();  // the next virtual block may reuse shared memory
    }
}

// The body of a kernel as a packable operation: SDR_OP(k_name, threads)
// declares k_name_op, whose run() calls k_name_body; `threads` is the largest
// block the call sites use.
#define SDR_OP(kern, threads)                                                   \
    struct kern##_op {                                                          \
        static constexpr int kThreads = (threads);                              \
        template <class... A>                                                   \
        __device__ __forceinline__ static void run(VB vb, A... a) {             \
            kern##_body(vb, a...);                                              \
        }                                                                       \
    };

// memset and copy as kernels (a copy may read or write pinned host memory,
// which the device addresses directly). Each virtual block handles 16 KiB.
constexpr size_t kPackChunk = 16384;
__device__ __forceinline__ void k_pack_memset_body(VB vb, unsigned char* p, int value, size_t bytes) {
    const size_t a = (size_t)vb.bid * kPackChunk, e = min(bytes, a + kPackChunk);
    const unsigned char v = (unsigned char)value;
    if ((((uintptr_t)p | a | e) & 15) == 0) {
        const uint32_t w = v * 0x01010101u;
        const uint4 q = make_uint4(w, w, w, w);
        for (size_t o = a + 16 * threadIdx.x; o < e; o += 16 * blockDim.x) *reinterpret_cast<uint4*>(p + o) = q;
    } else {
        for (size_t o = a + threadIdx.x; o < e; o += blockDim.x) p[o] = v;
    }
}
__device__ __forceinline__ void k_pack_copy_body(VB vb, unsigned char* d, const unsigned char* s, size_t bytes) {
    const size_t a = (size_t)vb.bid * kPackChunk, e = min(bytes, a + kPackChunk);
    if ((((uintptr_t)d | (uintptr_t)s | a | e) & 15) == 0) {
        for (size_t o = a + 16 * threadIdx.x; o < e; o += 16 * blockDim.x)
            *reinterpret_cast<uint4*>(d + o) = *reinterpret_cast<const uint4*>(s + o);
    } else {
        for (size_t o = a + threadIdx.x; o < e; o += blockDim.x) d[o] = s[o];
    }
}
SDR_OP(k_pack_memset, 256)
SDR_OP(k_pack_copy, 256)

// ---------------------------------------------------------------- host side
using PackLaunch = void (*)(const unsigned char* dev_hdr, unsigned grid, unsigned block, size_t smem,
                            cudaStream_t st);

using PackPrep = cudaError_t (*)(size_t smem);

template <class Op, class Tup>
void pack_launch(const unsigned char* dev_hdr, unsigned grid, unsigned block, size_t smem, cudaStream_t st) {
    k_packed<Op, Tup><<<grid, block, smem, st>>>(dev_hdr);
}
// Dynamic shared memory above the 48 KiB default (set before any capture).
template <class Op, class Tup>
cudaError_t pack_prep(size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(k_packed<Op, Tup>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// One launch of a packed step: its kernel, table (offset into the arena) and shape.
struct PackStep {
    PackLaunch fn;
    PackPrep prep;
    size_t hdr_at;
    unsigned grid, threads;
    size_t smem;
    bool operator==(const PackStep& o) const {
        return fn == o.fn && hdr_at == o.hdr_at && grid == o.grid && threads == o.threads && smem == o.smem;
    }
};

// One recorded operation of one scene.
struct PackEntry {
    int line, occ;        // call site and its repetition within the substep
    PackLaunch fn;        // the slot's batched kernel
    PackPrep prep;
    unsigned blocks, threads;
    size_t smem, align;
    std::vector<unsigned char> args;  // the argument tuple's bytes
};

class Packer {
   public:
    // A scene starts recording its substep.
    void begin_scene() {
        scenes_.emplace_back();
        occ_.clear();
    }

    template <class Op, class... A>
    void record(int line, unsigned blocks, unsigned threads, size_t smem, A... args) {
        using Tup = cuda::std::tuple<A...>;
        static_assert(std::is_trivially_copyable<Tup>::value, "packed arguments must be plain data");
        Tup t(args...);
        PackEntry e;
        e.line = line;
        e.occ = occ_[line]++;
        e.fn = &pack_launch<Op, Tup>;
        e.prep = &pack_prep<Op, Tup>;
        e.blocks = blocks;
        e.threads = threads;
        e.smem = smem;
        e.align = alignof(Tup);
        e.args.resize(sizeof(Tup));
        std::memcpy(e.args.data(), &t, sizeof(Tup));
        scenes_.back().push_back(std::move(e));
    }

    // Lay out every slot's table in the host arena and plan the launches,
    // one per slot, in order: grid = the slot's virtual blocks rounded up to a
    // power of two, at most grid_cap (the CTAs then walk the virtual blocks),
    // so the plan - and a graph captured from it - stays the same while the
    // scenes' work changes within those buckets. Clears the recordings.
    const std::vector<unsigned char>& build(unsigned grid_cap, std::vector<PackStep>& plan) {
        // slots: the union of the scenes' (line, occ) keys, each scene's order kept
        std::vector<std::pair<int, int>> order;
        std::map<std::pair<int, int>, size_t> where;
        for (auto& sc : scenes_) {
            size_t at = 0;  // insertion point after this scene's previous slot
            for (auto& e : sc) {
                auto key = std::make_pair(e.line, e.occ);
                auto it = where.find(key);
                if (it == where.end()) {
                    order.insert(order.begin() + (long)at, key);
                    where.clear();
                    for (size_t q = 0; q < order.size(); ++q) where[order[q]] = q;
                    at = where[key] + 1;
                } else {
                    at = std::max(at, it->second + 1);
                }
            }
        }
        // per slot: the scenes' entries in scene order
        std::vector<std::vector<const PackEntry*>> slot(order.size());
        for (auto& sc : scenes_)
            for (auto& e : sc) slot[where[std::make_pair(e.line, e.occ)]].push_back(&e);
        host_.clear();
        plan.clear();
        for (size_t q = 0; q < order.size(); ++q) {
            const auto& es = slot[q];
            align(256);
            const size_t hdr_at = host_.size();
            PackHdr h{};
            h.ns = (uint32_t)es.size();
            host_.resize(host_.size() + sizeof(PackHdr));
            h.off_at = (uint32_t)(host_.size() - hdr_at);
            uint32_t tot = 0;
            unsigned threads = 0;
            size_t smem = 0;
            for (auto* e : es) {
                push_u32(tot);
                tot += e->blocks;
                threads = std::max(threads, e->threads);
                smem = std::max(smem, e->smem);
            }
            push_u32(tot);
            h.total = tot;
            align(16);
            h.args_at = (uint32_t)(host_.size() - hdr_at);
            h.stride = (uint32_t)((es[0]->args.size() + 15) & ~(size_t)15);
            for (auto* e : es) {
                const size_t at = host_.size();
                host_.resize(at + h.stride, 0);
                std::memcpy(host_.data() + at, e->args.data(), e->args.size());
            }
            std::memcpy(host_.data() + hdr_at, &h, sizeof(h));
            unsigned grid = 1;
            while (grid < tot && grid < grid_cap) grid <<= 1;
            plan.push_back(PackStep{es[0]->fn, es[0]->prep, hdr_at, std::min(grid, grid_cap), threads, smem});
        }
        scenes_.clear();
        return host_;
    }

    // The last scene's recording is abandoned (it failed part way).
    void drop_scene() {
        if (!scenes_.empty()) scenes_.pop_back();
    }

    void clear() { scenes_.clear(); }

   private:
    void align(size_t a) { host_.resize((host_.size() + a - 1) / a * a, 0); }
    void push_u32(uint32_t v) {
        const size_t at = host_.size();
        host_.resize(at + 4);
        std::memcpy(host_.data() + at, &v, 4);
    }
    std::vector<std::vector<PackEntry>> scenes_;
    std::map<int, int> occ_;
    std::vector<unsigned char> host_;
};

}  // namespace sdr
