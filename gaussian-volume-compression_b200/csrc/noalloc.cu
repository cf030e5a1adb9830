// noalloc.cu -- tetrahedral mesh sampling without any device allocation.
//
// Some callers of this library cannot allocate device memory when they sample a mesh:
// an application whose device memory is owned by another allocator (a framework's
// caching allocator that has reserved the pool, or a host that forbids allocation after
// start-up), or a latency-critical loop where cudaMalloc / cudaFree would synchronise the
// whole device.  gvc_sample_tets_static() serves them: the caller passes inputs and
// outputs, and the only scratch (the cell LBVH and its sort buffers) lives in one
// file-scope device array of fixed size, held by every device that loads the library
// until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the array's
// device address with cudaGetSymbolAddress (the array's name is only a host-side
// stand-in in host code) and caches it for that device.  Under CUDA's default lazy
// module loading that lookup is also when the driver loads this library's device code
// on the device and reserves the array, so the first call per device does reserve
// device memory once; a call with N = 0 does only this set-up, and callers that must not
// allocate later make it at start-up (or run with CUDA_MODULE_LOADING=EAGER, which
// reserves the array when the library's device code loads).  That first call should
// come before any stream capture on the device.
//
// Every call returns after `stream` has finished the call's work: it reads the traversal
// status word back to the host.
//
// Every call shares the array and it keeps the last call's contents; whatever must
// start at zero is cleared on each call.  Calls whose work overlaps on the GPU (two
// streams, two threads) race on the array: issue them one after another.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "lbvh.cuh"
#include "render.cuh"

namespace {

constexpr int64_t kStaticMaxCells = 32768;
constexpr size_t kAlign = 256;

constexpr size_t up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// Regions carved out of the array for kStaticMaxCells cells, each sized by the LBVH
// builder's own rules (LbvhBytes) for that many boxes.
constexpr int64_t kC = kStaticMaxCells;
using gvc::LbvhBytes;
constexpr size_t kOffStatus = 0;
constexpr size_t kOffBoxes = kOffStatus + up(sizeof(int));
constexpr size_t kOffKeys = kOffBoxes + up(32 * kC);
constexpr size_t kOffKeysAlt = kOffKeys + up(LbvhBytes::keys(kC));
constexpr size_t kOffPerm = kOffKeysAlt + up(LbvhBytes::keys(kC));
constexpr size_t kOffPermAlt = kOffPerm + up(LbvhBytes::keys(kC));
constexpr size_t kOffHist = kOffPermAlt + up(LbvhBytes::keys(kC));
constexpr size_t kOffBounds = kOffHist + up(LbvhBytes::hist(kC));
constexpr size_t kOffSorted = kOffBounds + up(LbvhBytes::bounds());
constexpr size_t kOffLeft = kOffSorted + up(LbvhBytes::sorted_boxes(kC));
constexpr size_t kOffRight = kOffLeft + up(LbvhBytes::child(kC));
constexpr size_t kOffParent = kOffRight + up(LbvhBytes::child(kC));
constexpr size_t kOffFlags = kOffParent + up(LbvhBytes::parent(kC));
constexpr size_t kOffNodeBoxes = kOffFlags + up(LbvhBytes::child(kC));
constexpr size_t kOffNodes = kOffNodeBoxes + up(LbvhBytes::node_boxes(kC));
constexpr size_t kScratchBytes = kOffNodes + up(LbvhBytes::nodes(kC));  // about 6.4 MB
static_assert(kScratchBytes < (size_t(8) << 20), "the static scratch array is meant to stay modest");
static_assert(kOffBoxes % 16 == 0 && kOffSorted % 16 == 0 && kOffNodes % 64 == 0, "region alignment");

}  // namespace

// The scratch array (device memory of every device that loads libgvc.so).
static __device__ __align__(256) unsigned char g_tet_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 128;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

void set_msg(char* buf, int64_t len, const char* msg) {
    if (buf && len > 0) {
        std::strncpy(buf, msg, (size_t)len - 1);
        buf[len - 1] = '\0';
    }
}

gvc::DevBuf view(unsigned char* base, size_t off, size_t bytes) {
    gvc::DevBuf b;
    b.ptr = base + off;
    b.bytes = bytes;
    return b;
}

}  // namespace

extern "C" int gvc_sample_tets_static(int64_t npts, const float* pts, int64_t C, const int32_t* conn4,
                                      const double* values, int64_t N, const float* samples, double* out,
                                      int64_t* cell_ids, void* stream, char* errbuf, int64_t errbuf_len) {
    if (npts < 0 || C < 0 || N < 0) {
        set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: negative size");
        return GVC_ERR_ARG;
    }
    if (C > kStaticMaxCells) {
        char m[160];
        std::snprintf(m, sizeof(m), "gvc_sample_tets_static: %lld cells exceed the static maximum of %lld",
                      (long long)C, (long long)kStaticMaxCells);
        set_msg(errbuf, errbuf_len, m);
        return GVC_ERR_CAPACITY;
    }
    if (N > (int64_t(1) << 31) - 4096) {
        set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: too many sample points");
        return GVC_ERR_CAPACITY;
    }
    if (N > 0 && (!samples || !out)) {
        set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: null samples or output");
        return GVC_ERR_ARG;
    }
    if (C > 0 && (!pts || !conn4 || !values)) {
        set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: null mesh pointer");
        return GVC_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: no usable current device");
        return GVC_ERR_CUDA;
    }
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_tet_scratch);
            if (e != cudaSuccess || !p) {
                set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: cudaGetSymbolAddress failed");
                return GVC_ERR_CUDA;
            }
            g_scratch_addr[dev] = p;
        }
        base = static_cast<unsigned char*>(g_scratch_addr[dev]);
    }
    if (N == 0) return GVC_OK;  // set-up only
    cudaStream_t st = (cudaStream_t)stream;
    int* d_status = reinterpret_cast<int*>(base + kOffStatus);
    if ((e = cudaMemsetAsync(d_status, 0, sizeof(int), st)) != cudaSuccess) {
        set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: clearing the status word failed");
        return GVC_ERR_CUDA;
    }
    const gvc::BvhNode* cnodes = nullptr;
    const int32_t* cperm = nullptr;
    if (C > 0) {
        gvc::Lbvh L;  // views of the static array: every ensure() below fits, nothing is allocated
        L.keys = view(base, kOffKeys, LbvhBytes::keys(kC));
        L.keys_alt = view(base, kOffKeysAlt, LbvhBytes::keys(kC));
        L.perm = view(base, kOffPerm, LbvhBytes::keys(kC));
        L.perm_alt = view(base, kOffPermAlt, LbvhBytes::keys(kC));
        L.hist = view(base, kOffHist, LbvhBytes::hist(kC));
        L.bounds = view(base, kOffBounds, LbvhBytes::bounds());
        L.sorted_boxes = view(base, kOffSorted, LbvhBytes::sorted_boxes(kC));
        L.left = view(base, kOffLeft, LbvhBytes::child(kC));
        L.right = view(base, kOffRight, LbvhBytes::child(kC));
        L.parent = view(base, kOffParent, LbvhBytes::parent(kC));
        L.flags = view(base, kOffFlags, LbvhBytes::child(kC));
        L.node_boxes = view(base, kOffNodeBoxes, LbvhBytes::node_boxes(kC));
        L.nodes = view(base, kOffNodes, LbvhBytes::nodes(kC));
        // every view must hold what the builder asks for C boxes; then none of its
        // ensure() calls reallocates (an undersized view would be freed as if it were
        // allocated memory)
        const struct {
            const gvc::DevBuf& b;
            size_t need;
        } need[] = {{L.keys, LbvhBytes::keys(C)},          {L.keys_alt, LbvhBytes::keys(C)},
                    {L.perm, LbvhBytes::keys(C)},          {L.perm_alt, LbvhBytes::keys(C)},
                    {L.hist, LbvhBytes::hist(C)},          {L.bounds, LbvhBytes::bounds()},
                    {L.sorted_boxes, LbvhBytes::sorted_boxes(C)}, {L.left, LbvhBytes::child(C)},
                    {L.right, LbvhBytes::child(C)},        {L.parent, LbvhBytes::parent(C)},
                    {L.flags, LbvhBytes::child(C)},        {L.node_boxes, LbvhBytes::node_boxes(C)},
                    {L.nodes, LbvhBytes::nodes(C)}};
        for (const auto& r : need) {
            if (r.b.bytes < r.need) {
                set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: scratch layout too small");
                return GVC_ERR_CAPACITY;
            }
        }
        const void* before[] = {L.keys.ptr, L.keys_alt.ptr, L.perm.ptr, L.perm_alt.ptr, L.hist.ptr, L.bounds.ptr,
                                L.sorted_boxes.ptr, L.left.ptr, L.right.ptr, L.parent.ptr, L.flags.ptr,
                                L.node_boxes.ptr, L.nodes.ptr};
        float4* boxes = reinterpret_cast<float4*>(base + kOffBoxes);
        if ((e = gvc::launch_tet_boxes(C, pts, conn4, boxes, st)) != cudaSuccess ||
            (e = gvc::lbvh_build_boxes(L, C, boxes, st)) != cudaSuccess) {
            set_msg(errbuf, errbuf_len, cudaGetErrorString(e));
            return GVC_ERR_CUDA;
        }
        const void* after[] = {L.keys.ptr, L.keys_alt.ptr, L.perm.ptr, L.perm_alt.ptr, L.hist.ptr, L.bounds.ptr,
                               L.sorted_boxes.ptr, L.left.ptr, L.right.ptr, L.parent.ptr, L.flags.ptr,
                               L.node_boxes.ptr, L.nodes.ptr};
        if (std::memcmp(before, after, sizeof(before)) != 0) {  // a region was too small: never expected
            set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: scratch layout too small");
            return GVC_ERR_CAPACITY;
        }
        cnodes = L.nodes.as<gvc::BvhNode>();
        cperm = L.perm.as<int32_t>();
    }
    // samples are traversed in the caller's order (no per-sample scratch)
    if ((e = gvc::launch_sample_tets(N, samples, nullptr, pts, conn4, values, cnodes, cperm, C, out, cell_ids,
                                     d_status, st)) != cudaSuccess) {
        set_msg(errbuf, errbuf_len, cudaGetErrorString(e));
        return GVC_ERR_CUDA;
    }
    int h_status = 0;
    if ((e = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        set_msg(errbuf, errbuf_len, cudaGetErrorString(e));
        return GVC_ERR_CUDA;
    }
    if (h_status) {
        set_msg(errbuf, errbuf_len, "gvc_sample_tets_static: BVH traversal stack overflow");
        return GVC_ERR_TRAVERSAL;
    }
    return GVC_OK;
}
