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

// ---------------------------------------------------------------------------------
// General explicit cells: VTK_TETRA (10), VTK_HEXAHEDRON (12), VTK_WEDGE (13),
// VTK_PYRAMID (14) with isoparametric shape functions in VTK node order; the point is
// mapped to parametric coordinates by Newton's method in double (same expressions, same
// iteration rule as the oracle); zero-volume cells (1, 3, 5, 9) never contain a point.
// ---------------------------------------------------------------------------------
constexpr int kNewtonIters = 20;
constexpr double kNewtonTol = 1e-13;
constexpr double kInsideEps = 1e-9;

__device__ __forceinline__ int cell_npts(int type) {
    return type == 10 ? 4 : (type == 12 ? 8 : (type == 13 ? 6 : (type == 14 ? 5 : 0)));
}

__device__ int shape_eval(int type, double r, double s, double t, double N[8], double dN[8][3]) {
    if (type == 12) {
        const double rm = 1.0 - r, sm = 1.0 - s, tm = 1.0 - t;
        N[0] = rm * sm * tm; N[1] = r * sm * tm; N[2] = r * s * tm; N[3] = rm * s * tm;
        N[4] = rm * sm * t;  N[5] = r * sm * t;  N[6] = r * s * t;  N[7] = rm * s * t;
        dN[0][0] = -(sm * tm); dN[0][1] = -(rm * tm); dN[0][2] = -(rm * sm);
        dN[1][0] = sm * tm;    dN[1][1] = -(r * tm);  dN[1][2] = -(r * sm);
        dN[2][0] = s * tm;     dN[2][1] = r * tm;     dN[2][2] = -(r * s);
        dN[3][0] = -(s * tm);  dN[3][1] = rm * tm;    dN[3][2] = -(rm * s);
        dN[4][0] = -(sm * t);  dN[4][1] = -(rm * t);  dN[4][2] = rm * sm;
        dN[5][0] = sm * t;     dN[5][1] = -(r * t);   dN[5][2] = r * sm;
        dN[6][0] = s * t;      dN[6][1] = r * t;      dN[6][2] = r * s;
        dN[7][0] = -(s * t);   dN[7][1] = rm * t;     dN[7][2] = rm * s;
        return 8;
    }
    if (type == 13) {
        const double u = 1.0 - r - s, tm = 1.0 - t;
        N[0] = u * tm; N[1] = r * tm; N[2] = s * tm; N[3] = u * t; N[4] = r * t; N[5] = s * t;
        dN[0][0] = -tm; dN[0][1] = -tm; dN[0][2] = -u;
        dN[1][0] = tm;  dN[1][1] = 0.0; dN[1][2] = -r;
        dN[2][0] = 0.0; dN[2][1] = tm;  dN[2][2] = -s;
        dN[3][0] = -t;  dN[3][1] = -t;  dN[3][2] = u;
        dN[4][0] = t;   dN[4][1] = 0.0; dN[4][2] = r;
        dN[5][0] = 0.0; dN[5][1] = t;   dN[5][2] = s;
        return 6;
    }
    if (type == 14) {
        const double rm = 1.0 - r, sm = 1.0 - s, tm = 1.0 - t;
        N[0] = rm * sm * tm; N[1] = r * sm * tm; N[2] = r * s * tm; N[3] = rm * s * tm; N[4] = t;
        dN[0][0] = -(sm * tm); dN[0][1] = -(rm * tm); dN[0][2] = -(rm * sm);
        dN[1][0] = sm * tm;    dN[1][1] = -(r * tm);  dN[1][2] = -(r * sm);
        dN[2][0] = s * tm;     dN[2][1] = r * tm;     dN[2][2] = -(r * s);
        dN[3][0] = -(s * tm);  dN[3][1] = rm * tm;    dN[3][2] = -(rm * s);
        dN[4][0] = 0.0;        dN[4][1] = 0.0;        dN[4][2] = 1.0;
        return 5;
    }
    return 0;
}

__device__ int iso_contains(int type, const float* __restrict__ pts, const int32_t* __restrict__ cv, const float* p,
                            double Nout[8]) {
    double r, s, t;
    if (type == 12) { r = 0.5; s = 0.5; t = 0.5; }
    else if (type == 13) { r = 1.0 / 3.0; s = 1.0 / 3.0; t = 0.5; }
    else { r = 0.5; s = 0.5; t = 0.25; }
    double N[8], dN[8][3];
    int n = 0;
    bool converged = false;
    for (int it = 0; it < kNewtonIters; it++) {
        n = shape_eval(type, r, s, t, N, dN);
        double f[3] = {0.0, 0.0, 0.0}, J[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        for (int k = 0; k < n; k++) {
            const float* x = pts + 3 * (int64_t)cv[k];
            for (int a = 0; a < 3; a++) {
                f[a] = f[a] + N[k] * (double)x[a];
                for (int b = 0; b < 3; b++) J[a][b] = J[a][b] + dN[k][b] * (double)x[a];
            }
        }
        for (int a = 0; a < 3; a++) f[a] = f[a] - (double)p[a];
        const double det = det3(J[0][0], J[0][1], J[0][2], J[1][0], J[1][1], J[1][2], J[2][0], J[2][1], J[2][2]);
        if (det == 0.0 || det != det) return 0;
        const double d0 = det3(f[0], J[0][1], J[0][2], f[1], J[1][1], J[1][2], f[2], J[2][1], J[2][2]) / det;
        const double d1 = det3(J[0][0], f[0], J[0][2], J[1][0], f[1], J[1][2], J[2][0], f[2], J[2][2]) / det;
        const double d2 = det3(J[0][0], J[0][1], f[0], J[1][0], J[1][1], f[1], J[2][0], J[2][1], f[2]) / det;
        r = r - d0;
        s = s - d1;
        t = t - d2;
        double m = fabs(d0);
        if (fabs(d1) > m) m = fabs(d1);
        if (fabs(d2) > m) m = fabs(d2);
        if (!(m >= kNewtonTol)) {
            converged = true;
            break;
        }
    }
    // an unconverged iterate says nothing about the point: not contained
    if (!converged) return 0;
    const double e = kInsideEps;
    bool inside;
    if (type == 13) inside = r >= -e && s >= -e && r + s <= 1.0 + e && t >= -e && t <= 1.0 + e;
    else inside = r >= -e && r <= 1.0 + e && s >= -e && s <= 1.0 + e && t >= -e && t <= 1.0 + e;
    if (!inside) return 0;
    n = shape_eval(type, r, s, t, N, dN);
    for (int k = 0; k < n; k++) Nout[k] = N[k];
    return n;
}

__global__ void __launch_bounds__(256) k_cell_boxes(int64_t C, const float* __restrict__ pts,
                                                    const uint8_t* __restrict__ types,
                                                    const int64_t* __restrict__ offsets,
                                                    const int32_t* __restrict__ conn, float4* __restrict__ boxes) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= C) return;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int n = cell_npts(types[c]);
    for (int k = 0; k < n; k++) {
        const float* v = pts + 3 * (int64_t)conn[offsets[c] + k];
        for (int a = 0; a < 3; a++) {
            lo[a] = fminf(lo[a], v[a]);
            hi[a] = fmaxf(hi[a], v[a]);
        }
    }
    boxes[2 * c] = make_float4(lo[0], lo[1], lo[2], 0.f);
    boxes[2 * c + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
}

__global__ void __launch_bounds__(128) k_sample_cells(int64_t N, const float* __restrict__ samples,
                                                      const int32_t* __restrict__ sperm, const float* __restrict__ pts,
                                                      const uint8_t* __restrict__ types,
                                                      const int64_t* __restrict__ offsets,
                                                      const int32_t* __restrict__ conn,
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
                    const int type = types[cell];
                    const int32_t* cv = conn + offsets[cell];
                    if (type == 10) {
                        double lam[4];
                        if (tet_contains(pts + 3 * (int64_t)cv[0], pts + 3 * (int64_t)cv[1],
                                         pts + 3 * (int64_t)cv[2], pts + 3 * (int64_t)cv[3], p, lam)) {
                            double v = lam[0] * values[cv[0]];
                            v = v + lam[1] * values[cv[1]];
                            v = v + lam[2] * values[cv[2]];
                            v = v + lam[3] * values[cv[3]];
                            best = cell;
                            best_v = v;
                        }
                    } else if (type == 12 || type == 13 || type == 14) {
                        double Nf[8];
                        const int n = iso_contains(type, pts, cv, p, Nf);
                        if (n) {
                            double v = Nf[0] * values[cv[0]];
                            for (int q = 1; q < n; q++) v = v + Nf[q] * values[cv[q]];
                            best = cell;
                            best_v = v;
                        }
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

cudaError_t launch_cell_boxes(int64_t C, const float* pts, const uint8_t* types, const int64_t* offsets,
                              const int32_t* conn, float4* boxes, cudaStream_t st) {
    if (C <= 0) return cudaSuccess;
    k_cell_boxes<<<nbk(C, 256), 256, 0, st>>>(C, pts, types, offsets, conn, boxes); gvc::note_launch();
    return cudaGetLastError();
}

cudaError_t launch_sample_cells(int64_t N, const float* samples, const int32_t* sperm, const float* pts,
                                const uint8_t* types, const int64_t* offsets, const int32_t* conn,
                                const double* values, const BvhNode* cnodes, const int32_t* cperm, int64_t C,
                                double* out, int64_t* cell_ids, int* status, cudaStream_t st) {
    if (N <= 0) return cudaSuccess;
    k_sample_cells<<<nbk(N, 128), 128, 0, st>>>(N, samples, sperm, pts, types, offsets, conn, values, cnodes, cperm,
                                                C, out, cell_ids, status); gvc::note_launch();
    return cudaGetLastError();
}

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
