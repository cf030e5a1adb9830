// mesh.cu -- point sampling of structured (uniform) and tetrahedral meshes.
//
// Replaces the Viskores Probe filter calls of gpu_sampling/sample_mesh.cu:155-167
// (uniform point field) and :380-390 (explicit cells).  Compiled with --fmad=false:
// the double-precision locate / interpolate arithmetic rounds after every operation,
// as the oracle does, so cell ids and values are reproducible bit for bit.
//
// Declared semantics (the reference's Viskores internals are not vendored):
//   uniform: f = (x - o) / sp per axis; inside iff 0 <= f <= n-1; cell
//            i = min(floor(f), n-2); trilinear lerp a + t (b - a) along x, y, z;
//            outside -> -1 converted to the value dtype.
//   tets:    orient(a,b,c,d) = det[b-a, c-a, d-a]; closed containment by sub-volume
//            signs; degenerate tets never contain; ties -> lowest cell id;
//            value = sum_k (V_k / V) f_k; outside -> -1, cell -1.
#include "render.cuh"
#include "traverse.cuh"

namespace gvc {

template <class T>
__device__ __forceinline__ double ld_val(const void* v, int64_t i) {
    return (double)reinterpret_cast<const T*>(v)[i];
}

__device__ __forceinline__ double load_value(const void* v, int dtype, int64_t i) {
    switch (dtype) {
        case GVC_F64: return ld_val<double>(v, i);
        case GVC_F32: return ld_val<float>(v, i);
        case GVC_U16: return ld_val<uint16_t>(v, i);
        default: return ld_val<uint8_t>(v, i);
    }
}

// Integer outputs round half up and saturate; invalid (-1) wraps like a C cast of -1
// to the unsigned type (255 / 65535).
__device__ __forceinline__ void store_value(void* out, int dtype, int64_t i, double v, bool valid) {
    switch (dtype) {
        case GVC_F64: reinterpret_cast<double*>(out)[i] = valid ? v : -1.0; break;
        case GVC_F32: reinterpret_cast<float*>(out)[i] = valid ? (float)v : -1.0f; break;
        case GVC_U16: {
            uint16_t r = 0xffffu;
            if (valid) {
                double t = floor(v + 0.5);
                r = t <= 0.0 ? 0u : (t >= 65535.0 ? 65535u : (uint16_t)t);
            }
            reinterpret_cast<uint16_t*>(out)[i] = r;
            break;
        }
        default: {
            uint8_t r = 0xffu;
            if (valid) {
                double t = floor(v + 0.5);
                r = t <= 0.0 ? 0u : (t >= 255.0 ? 255u : (uint8_t)t);
            }
            reinterpret_cast<uint8_t*>(out)[i] = r;
        }
    }
}

struct UniformGrid {
    int64_t n[3];
    float o[3], sp[3];
};

__device__ __forceinline__ double lerp_d(double a, double b, double t) { return a + t * (b - a); }

__global__ void __launch_bounds__(256) k_sample_uniform(UniformGrid g, const void* __restrict__ values, int dtype,
                                                        int64_t N, const float* __restrict__ samples, void* out) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= N) return;
    int64_t ci[3];
    double t[3];
    bool ok = true;
    for (int a = 0; a < 3; a++) {
        const double f = ((double)samples[3 * s + a] - (double)g.o[a]) / (double)g.sp[a];
        const int64_t n = g.n[a];
        if (!(f >= 0.0) || !(f <= (double)(n - 1))) {
            ok = false;
            break;
        }
        if (n == 1) {
            ci[a] = 0;
            t[a] = 0.0;
            continue;
        }
        int64_t i = (int64_t)floor(f);
        if (i > n - 2) i = n - 2;
        ci[a] = i;
        t[a] = f - (double)i;
    }
    if (!ok) {
        store_value(out, dtype, s, 0.0, false);
        return;
    }
    const int64_t nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int64_t sx = nx > 1 ? 1 : 0, sy = ny > 1 ? nx : 0, sz = nz > 1 ? nx * ny : 0;
    const int64_t b = ci[0] + nx * (ci[1] + ny * ci[2]);
    const double v000 = load_value(values, dtype, b), v100 = load_value(values, dtype, b + sx);
    const double v010 = load_value(values, dtype, b + sy), v110 = load_value(values, dtype, b + sx + sy);
    const double v001 = load_value(values, dtype, b + sz), v101 = load_value(values, dtype, b + sx + sz);
    const double v011 = load_value(values, dtype, b + sy + sz), v111 = load_value(values, dtype, b + sx + sy + sz);
    const double c00 = lerp_d(v000, v100, t[0]), c10 = lerp_d(v010, v110, t[0]);
    const double c01 = lerp_d(v001, v101, t[0]), c11 = lerp_d(v011, v111, t[0]);
    const double c0 = lerp_d(c00, c10, t[1]), c1 = lerp_d(c01, c11, t[1]);
    store_value(out, dtype, s, lerp_d(c0, c1, t[2]), true);
}

// ---------------------------------------------------------------------------------
// Tetrahedra
// ---------------------------------------------------------------------------------
__device__ __forceinline__ double det3(double ux, double uy, double uz, double vx, double vy, double vz, double wx,
                                       double wy, double wz) {
    const double m0 = vy * wz - vz * wy;
    const double m1 = vx * wz - vz * wx;
    const double m2 = vx * wy - vy * wx;
    double r = ux * m0;
    r = r - uy * m1;
    r = r + uz * m2;
    return r;
}

__device__ __forceinline__ double orient(const float* a, const float* b, const float* c, const float* d) {
    const double ax = a[0], ay = a[1], az = a[2];
    return det3((double)b[0] - ax, (double)b[1] - ay, (double)b[2] - az, (double)c[0] - ax, (double)c[1] - ay,
                (double)c[2] - az, (double)d[0] - ax, (double)d[1] - ay, (double)d[2] - az);
}

__device__ __forceinline__ bool tet_contains(const float* a, const float* b, const float* c, const float* d,
                                             const float* p, double lam[4]) {
    const double V = orient(a, b, c, d);
    if (V == 0.0) return false;
    const double Va = orient(p, b, c, d), Vb = orient(a, p, c, d), Vc = orient(a, b, p, d), Vd = orient(a, b, c, p);
    if (V > 0) {
        if (Va < 0 || Vb < 0 || Vc < 0 || Vd < 0) return false;
    } else {
        if (Va > 0 || Vb > 0 || Vc > 0 || Vd > 0) return false;
    }
    lam[0] = Va / V;
    lam[1] = Vb / V;
    lam[2] = Vc / V;
    lam[3] = Vd / V;
    return true;
}

__global__ void __launch_bounds__(256) k_tet_boxes(int64_t C, const float* __restrict__ pts,
                                                   const int32_t* __restrict__ conn4, float4* __restrict__ boxes) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= C) return;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < 4; k++) {
        const float* v = pts + 3 * (int64_t)conn4[4 * c + k];
        for (int a = 0; a < 3; a++) {
            lo[a] = fminf(lo[a], v[a]);
            hi[a] = fmaxf(hi[a], v[a]);
        }
    }
    boxes[2 * c] = make_float4(lo[0], lo[1], lo[2], 0.f);
    boxes[2 * c + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
}

constexpr int kPointStack = 96;

// One thread per (Morton-sorted) sample; point query of the cell LBVH with a
// per-thread stack; every containing tet is tested and the lowest id kept.
__global__ void __launch_bounds__(128) k_sample_tets(int64_t N, const float* __restrict__ samples,
                                                     const int32_t* __restrict__ sperm, const float* __restrict__ pts,
                                                     const int32_t* __restrict__ conn4,
                                                     const double* __restrict__ values,
                                                     const BvhNode* __restrict__ nodes,
                                                     const int32_t* __restrict__ cperm, int64_t C,
                                                     double* __restrict__ out, int64_t* __restrict__ cell_ids,
                                                     int* status) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int64_t s = sperm ? sperm[i] : i;
    const float p[3] = {samples[3 * s], samples[3 * s + 1], samples[3 * s + 2]};
    int64_t best = -1;
    double best_v = -1.0;
    if (C > 0) {
        int stack[kPointStack];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const int node = stack[--sp];
            const float4* np = reinterpret_cast<const float4*>(nodes + node);
            const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2), d = __ldg(np + 3);
            const uint32_t ch[2] = {__float_as_uint(a.w), __float_as_uint(b.w)};
            const bool hit[2] = {a.x <= p[0] && p[0] <= b.x && a.y <= p[1] && p[1] <= b.y && a.z <= p[2] && p[2] <= b.z,
                                 c.x <= p[0] && p[0] <= d.x && c.y <= p[1] && p[1] <= d.y && c.z <= p[2] && p[2] <= d.z};
            for (int k = 0; k < 2; k++) {
                if (!hit[k]) continue;
                if (ch[k] & kLeafBit) {
                    const int64_t cell = cperm[ch[k] & ~kLeafBit];
                    if (best >= 0 && cell > best) continue;
                    const int32_t* cv = conn4 + 4 * cell;
                    double lam[4];
                    if (tet_contains(pts + 3 * (int64_t)cv[0], pts + 3 * (int64_t)cv[1], pts + 3 * (int64_t)cv[2],
                                     pts + 3 * (int64_t)cv[3], p, lam)) {
                        double v = lam[0] * values[cv[0]];
                        v = v + lam[1] * values[cv[1]];
                        v = v + lam[2] * values[cv[2]];
                        v = v + lam[3] * values[cv[3]];
                        best = cell;
                        best_v = v;
                    }
                } else if (sp < kPointStack) {
                    stack[sp++] = (int)ch[k];
                } else {
                    atomicOr(status, kStatusStackOverflow);
                }
            }
        }
    }
    out[s] = best >= 0 ? best_v : -1.0;
    if (cell_ids) cell_ids[s] = best;
}

static inline unsigned nbk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t launch_sample_uniform(const int64_t dims[3], const float origin[3], const float spacing[3],
                                  const void* values, int dtype, int64_t N, const float* samples, void* out,
                                  cudaStream_t st) {
    if (N <= 0) return cudaSuccess;
    UniformGrid g;
    for (int a = 0; a < 3; a++) {
        g.n[a] = dims[a];
        g.o[a] = origin[a];
        g.sp[a] = spacing[a];
    }
    k_sample_uniform<<<nbk(N, 256), 256, 0, st>>>(g, values, dtype, N, samples, out); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_tet_boxes(int64_t C, const float* pts, const int32_t* conn4, float4* boxes, cudaStream_t st) {
    if (C <= 0) return cudaSuccess;
    k_tet_boxes<<<nbk(C, 256), 256, 0, st>>>(C, pts, conn4, boxes); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_sample_tets(int64_t N, const float* samples, const int32_t* sperm, const float* pts,
                               const int32_t* conn4, const double* values, const BvhNode* cnodes,
                               const int32_t* cperm, int64_t C, double* out, int64_t* cell_ids, int* status,
                               cudaStream_t st) {
    if (N <= 0) return cudaSuccess;
    k_sample_tets<<<nbk(N, 128), 128, 0, st>>>(N, samples, sperm, pts, conn4, values, cnodes, cperm, C, out,
                                               cell_ids, status); gvc::note_launch();
    return cudaGetLastError();
}

}  // namespace gvc
