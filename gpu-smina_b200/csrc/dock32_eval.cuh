// Mixed-precision path, part 1: one warp, or a team of warps that share out
// the grid and pair terms, evaluates model::eval_deriv in FP32.
//
// Energy, gradient and torsion-tree math run in FP32; the conf (position,
// orientation quaternion, torsions) stays in FP64 and is narrowed when the
// tree is set.  Grid maps are read in the packed-corner layout (one 32 B or
// 16 B load per atom); a pair interpolation is one float4 table load.
// Reference semantics: model.cpp:837-841,904-928,969-985; grid.cpp:111-236;
// tree.h:108-243; precalculate.h:111-151.
#pragma once
#include "sg_dev.cuh"

namespace sg {

constexpr unsigned kFull32 = 0xffffffffu;

// Loops that are run a handful of times per evaluation are kept rolled by
// default: the evaluation is latency-bound and instruction-cache-bound, so
// shorter code beats unrolled code there.
#ifndef SG_UNROLL_HOT
#define SG_ROLLED _Pragma("unroll 1")
#else
#define SG_ROLLED
#endif

#ifndef SG_PAIR_CHUNKS
#define SG_PAIR_CHUNKS 3  // pair chunks (of 32) whose table loads are in flight together
#endif

// Section timers (compile with -DSG_PROFILE): lane 0 of every warp adds
// clock64() spans per section; sg_profile_read() copies them out.
// Sections: 0 set_conf, 1 grid, 2 pairs, 3 derivative, 4 line-search
// bookkeeping, 5 BFGS algebra, 6 mutation, 7 whole chain, 8 wait at the
// block barrier after a work item.
#ifdef SG_PROFILE
__device__ unsigned long long g_prof[16];
#define SG_T0(name) const long long name = clock64()
#define SG_T1(name, k) \
    if ((threadIdx.x & 31) == 0) atomicAdd(&g_prof[k], (unsigned long long)(clock64() - name))
#else
#define SG_T0(name)
#define SG_T1(name, k)
#endif

// Dynamic shared memory of the mixed-precision kernels: the block's staged
// model (SModel + arrays) at offset 0, then one workspace per warp.  Every
// access is this symbol plus a 32-bit offset, so it compiles to shared-space
// loads and stores with 32-bit addresses.
extern __shared__ __align__(16) char smem32[];
__shared__ DTables32 sT32;  // the pair table descriptor of the running kernel
__shared__ DMaps32 sG32;    // the grid maps of the running kernel

template <typename T>
__device__ __forceinline__ T* sp(int off) {
    return reinterpret_cast<T*>(smem32 + off);
}
__device__ __forceinline__ const SModel& smodel() { return *reinterpret_cast<const SModel*>(smem32); }

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw 2011) -------------------------------
struct Philox {
    uint32_t k0, k1;  // key: request seed
    uint32_t c2, c3;  // counter words fixed per chain: (ligand, chain)
    uint32_t n;       // draw index
};
__device__ __forceinline__ uint4 philox10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}
// uniform double in [0, 1) with 53 random bits; every lane computes the same
// value.  Out of line: one copy of the ten rounds serves every draw site.
// The state is passed by value so that callers keep it in registers.
__device__ __noinline__ double ph_u01_at(uint32_t n, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    const uint4 o = philox10(make_uint4(n, 0u, c2, c3), k0, k1);
    const uint64_t v = ((uint64_t)(o.x >> 5) << 26) | (o.y >> 6);
    return (double)v * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ double ph_u01(Philox& r) { return ph_u01_at(r.n++, r.c2, r.c3, r.k0, r.k1); }
__device__ __forceinline__ double ph_range(Philox& r, double a, double b) { return a + (b - a) * ph_u01(r); }
__device__ __forceinline__ int ph_int(Philox& r, int n) {  // [0, n)
    const int k = (int)(ph_u01(r) * n);
    return k < n ? k : n - 1;
}
__device__ __forceinline__ double ph_normal(Philox& r) {  // Box-Muller
    const double u1 = 1.0 - ph_u01(r), u2 = ph_u01(r);
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// This warp's workspace: its byte offset in smem32 and the lane.  The
// layout is the block's (SModel::L).  Every function builds it on the spot
// from threadIdx and two block constants, so it lives in registers.
__shared__ int sWs0, sWsStride;  // first warp's workspace offset, stride between warps
struct W32 {
    int ws, lane;
    __device__ int at(int field) const { return ws + field; }  // smem32 offset of a workspace array
    __device__ float4* coords() const { return sp<float4>(ws + smodel().L.coords); }
    __device__ float4* force() const { return sp<float4>(ws + smodel().L.force); }
    __device__ float4* origin() const { return sp<float4>(ws + smodel().L.origin); }
    __device__ float4* axis() const { return sp<float4>(ws + smodel().L.axis); }
    __device__ float4* quat() const { return sp<float4>(ws + smodel().L.quat); }
    __device__ float4* rot() const { return sp<float4>(ws + smodel().L.rot); }
    __device__ double* d(int field) const { return sp<double>(ws + field); }
    // work counters: grid lookups per lane [0, 32), in-cutoff pair lookups
    // per lane [32, 64), evaluations [64]
    __device__ unsigned* counters() const { return sp<unsigned>(ws + smodel().L.scratch); }
};
__device__ __forceinline__ W32 here() {
    return W32{sWs0 + (int)(threadIdx.x >> 5) * sWsStride, (int)(threadIdx.x & 31)};
}

// the device's nanosecond clock (%globaltimer), comparable across launches
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 rot_apply(const float4* R, float3 v) {  // rows R[0..2]
    return make_float3(R[0].x * v.x + R[0].y * v.y + R[0].z * v.z, R[1].x * v.x + R[1].y * v.y + R[1].z * v.z,
                       R[2].x * v.x + R[2].y * v.y + R[2].z * v.z);
}
__device__ __forceinline__ void quat_rows(float4 q, float4* R) {
    const float a = q.x, b = q.y, c = q.z, d = q.w;
    const float aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c, bd = b * d, cc = c * c,
                cd = c * d, dd = d * d;
    R[0] = make_float4(aa + bb - cc - dd, 2 * (-ad + bc), 2 * (ac + bd), 0);
    R[1] = make_float4(2 * (ad + bc), aa - bb + cc - dd, 2 * (-ab + cd), 0);
    R[2] = make_float4(2 * (-ac + bd), 2 * (ab + cd), aa - bb - cc + dd, 0);
}
__device__ __forceinline__ float4 qmul32(float4 l, float4 r) {
    return make_float4(l.x * r.x - l.y * r.y - l.z * r.z - l.w * r.w, l.x * r.y + l.y * r.x + l.z * r.w - l.w * r.z,
                       l.x * r.z - l.y * r.w + l.z * r.x + l.w * r.y, l.x * r.w + l.y * r.z - l.z * r.y + l.w * r.x);
}
// rotate v by unit quaternion q = (w; x, y, z)
__device__ __forceinline__ float3 qrot(float4 q, float3 v) {
    const float3 u = make_float3(q.y, q.z, q.w);
    const float3 t = 2.0f * cross3(u, v);
    return v + q.x * t + cross3(u, t);
}
__device__ __forceinline__ float4 axis_angle32(float3 ax, float angle) {
    // bring the angle into [-pi, pi] (normalize_angle) before halving it
    const float twopi = 6.28318530717958647692f;
    angle -= twopi * rintf(angle * (1.0f / twopi));
    float s, c;
    __sincosf(0.5f * angle, &s, &c);
    return make_float4(c, s * ax.x, s * ax.y, s * ax.z);
}
__device__ __forceinline__ float4 q_norm_approx32(float4 q) {
    const float s = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (fabsf(s - 1.f) < 1e-6f) return q;
    const float inv = rsqrtf(s);
    return make_float4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull32, v, o);
    return v;
}


// model::set frame by frame, level after level (trees of more than 32
// frames); out of line because typical ligands never need it
__device__ __noinline__ void set_frames_by_level(W32 w, const double* conf) {
    const SModel& m = smodel();
    const int* fkind = sp<const int>(m.fkind);
    const int* fconf = sp<const int>(m.fconf);
    const int* fparent = sp<const int>(m.fparent);
    const float4* forigin = sp<const float4>(m.forigin32);
    const float4* faxis = sp<const float4>(m.faxis32);
    float4* O = w.origin();
    float4* A = w.axis();
    float4* Q = w.quat();
    float4* R = w.rot();
    for (int lv = 0; lv < m.nlevels; lv++) {
        for (int idx = __ldcg(m.level_start + lv) + w.lane; idx < __ldcg(m.level_start + lv + 1); idx += 32) {
            const int f = __ldcg(m.level_frames + idx);
            const int kind = fkind[f];
            float4 q;
            if (kind == SG_FRAME_RIGID) {
                const double* c = conf + fconf[f];
                O[f] = make_float4((float)c[0], (float)c[1], (float)c[2], 0);
                q = make_float4((float)c[3], (float)c[4], (float)c[5], (float)c[6]);
            } else if (kind == SG_FRAME_SEGMENT) {
                const int p = fparent[f];
                const float3 o = f3(O[p]) + rot_apply(R + 3 * p, f3(forigin[f]));
                const float3 ax = rot_apply(R + 3 * p, f3(faxis[f]));
                O[f] = make_float4(o.x, o.y, o.z, 0);
                A[f] = make_float4(ax.x, ax.y, ax.z, 0);
                q = q_norm_approx32(qmul32(axis_angle32(ax, (float)conf[fconf[f]]), Q[p]));
            } else {
                const float3 ax = f3(faxis[f]);
                O[f] = forigin[f];
                A[f] = make_float4(ax.x, ax.y, ax.z, 0);
                q = axis_angle32(ax, (float)conf[fconf[f]]);
            }
            Q[f] = q;
            quat_rows(q, R + 3 * f);
        }
        __syncwarp();
    }
}

// model::set in FP32.  Each frame's transform relative to its parent is a
// rotation about its parent-frame axis plus its parent-frame origin offset:
// turning about the lab axis R_p a equals R_p turning about a, so
// q_f = q_p r(a_f, theta_f) and o_f = o_p + R_p t_f.  These local transforms
// need no parent data; the lab transforms are their ordered compositions
// along the path to the root, done by pointer jumping in log2(depth) warp
// shuffles.  Trees of more than 32 frames go level by level.
__device__ __noinline__ void set_conf32(int conf_at) {
    const W32 w = here();
    const SModel& m = smodel();
    const double* conf = sp<const double>(conf_at);
    const int nframes = m.nframes, nmov = m.nmov;
    const int* fkind = sp<const int>(m.fkind);
    const int* fconf = sp<const int>(m.fconf);
    const int* fparent = sp<const int>(m.fparent);
    const float4* forigin = sp<const float4>(m.forigin32);
    const float4* faxis = sp<const float4>(m.faxis32);
    float4* O = w.origin();
    float4* A = w.axis();
    float4* Q = w.quat();
    float4* R = w.rot();
    if (nframes <= 32) {
        const int f = w.lane;
        const bool act = f < nframes;
        float4 q = make_float4(1, 0, 0, 0);
        float3 t = make_float3(0, 0, 0);
        int anc = -1, parent = -1, kind = 0;
        if (act) {
            kind = fkind[f];
            const int ci = fconf[f];
            if (kind == SG_FRAME_RIGID) {
                const double* c = conf + ci;
                t = make_float3((float)c[0], (float)c[1], (float)c[2]);
                q = make_float4((float)c[3], (float)c[4], (float)c[5], (float)c[6]);
            } else {
                if (kind == SG_FRAME_SEGMENT) parent = anc = fparent[f];
                t = f3(forigin[f]);
                q = axis_angle32(f3(faxis[f]), (float)conf[ci]);
            }
        }
        SG_ROLLED
        for (int it = 0; it < 6 && __any_sync(kFull32, anc >= 0); it++) {
            const int src = anc >= 0 ? anc : f;
            const float qa0 = __shfl_sync(kFull32, q.x, src), qa1 = __shfl_sync(kFull32, q.y, src),
                        qa2 = __shfl_sync(kFull32, q.z, src), qa3 = __shfl_sync(kFull32, q.w, src);
            const float ta0 = __shfl_sync(kFull32, t.x, src), ta1 = __shfl_sync(kFull32, t.y, src),
                        ta2 = __shfl_sync(kFull32, t.z, src);
            const int aa = __shfl_sync(kFull32, anc, src);
            if (anc >= 0) {
                const float4 qa = make_float4(qa0, qa1, qa2, qa3);
                t = make_float3(ta0, ta1, ta2) + qrot(qa, t);
                q = qmul32(qa, q);
                anc = aa;
            }
        }
        q = q_norm_approx32(q);
        // lab axis of a segment: its relative axis turned by the parent's orientation
        const int ps = parent >= 0 ? parent : f;
        const float4 pq = make_float4(__shfl_sync(kFull32, q.x, ps), __shfl_sync(kFull32, q.y, ps),
                                      __shfl_sync(kFull32, q.z, ps), __shfl_sync(kFull32, q.w, ps));
        if (act) {
            O[f] = make_float4(t.x, t.y, t.z, 0);
            Q[f] = q;
            quat_rows(q, R + 3 * f);
            if (kind == SG_FRAME_SEGMENT) {
                const float3 ax = qrot(pq, f3(faxis[f]));
                A[f] = make_float4(ax.x, ax.y, ax.z, 0);
            } else if (kind == SG_FRAME_FIRST_SEGMENT) {
                A[f] = faxis[f];
            }
        }
        __syncwarp();
    } else {
        set_frames_by_level(w, conf);
    }
    float4* X = w.coords();
    const int* atom_frame = sp<const int>(m.atom_frame);
    const float4* local = sp<const float4>(m.local32);
    for (int i = w.lane; i < nmov; i += 32) {
        const int f = atom_frame[i];
        const float3 c = f3(O[f]) + rot_apply(R + 3 * f, f3(local[i]));
        X[i] = make_float4(c.x, c.y, c.z, 0);
    }
    __syncwarp();
}

// grid::evaluate_aux on the packed-corner map
__device__ __forceinline__ float grid_aux32(const DMaps32& G, int t, bool charge_map, float3 loc, float slope, float v,
                                            float3& deriv) {
    float s[3] = {(loc.x - G.init[0]) * G.factor[0], (loc.y - G.init[1]) * G.factor[1], (loc.z - G.init[2]) * G.factor[2]};
    float miss[3] = {0, 0, 0};
    int region[3], a[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (s[i] < 0) { miss[i] = -s[i]; region[i] = -1; a[i] = 0; s[i] = 0; }
        else if (s[i] >= G.dim_fl_minus_1[i]) { miss[i] = s[i] - G.dim_fl_minus_1[i]; region[i] = 1; a[i] = G.cdim[i] - 1; s[i] = 1; }
        else { region[i] = 0; a[i] = min((int)s[i], G.cdim[i] - 1); s[i] -= (float)a[i]; }
    }
    const float penalty = slope * (miss[0] * G.factor_inv[0] + miss[1] * G.factor_inv[1] + miss[2] * G.factor_inv[2]);
    const int cell = a[0] + G.cdim[0] * (a[1] + G.cdim[1] * a[2]);
    float4 lo, hi;
    if (!charge_map && G.half) {
        const uint4 u = __ldg(G.m16[t] + cell);
        const float2 p0 = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
        const float2 p1 = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
        const float2 p2 = __half22float2(*reinterpret_cast<const __half2*>(&u.z));
        const float2 p3 = __half22float2(*reinterpret_cast<const __half2*>(&u.w));
        lo = make_float4(p0.x, p0.y, p1.x, p1.y);
        hi = make_float4(p2.x, p2.y, p3.x, p3.y);
    } else {
        const float4* b = (charge_map ? G.c32[t] : G.m32[t]) + 2 * cell;
        lo = __ldg(b);
        hi = __ldg(b + 1);
    }
    const float x = s[0], y = s[1], z = s[2], mx = 1 - x, my = 1 - y, mz = 1 - z;
    // lo = (f000 f100 f010 f110), hi = (f001 f101 f011 f111)
    const float e00 = lo.x * mx + lo.y * x, e10 = lo.z * mx + lo.w * x;
    const float e01 = hi.x * mx + hi.y * x, e11 = hi.z * mx + hi.w * x;
    const float ez0 = e00 * my + e10 * y, ez1 = e01 * my + e11 * y;
    float f = ez0 * mz + ez1 * z;
    const float dx0 = (lo.y - lo.x) * my + (lo.w - lo.z) * y, dx1 = (hi.y - hi.x) * my + (hi.w - hi.z) * y;
    float3 grad = make_float3(dx0 * mz + dx1 * z, (e10 - e00) * mz + (e11 - e01) * z, ez1 - ez0);
    if (f > 0) {  // soft curl
        const float tt = (v < 1.1920929e-07f) ? 0.f : __fdividef(v, v + f);
        f *= tt;
        grad = (tt * tt) * grad;
    }
    deriv.x = G.factor[0] * (region[0] == 0 ? grad.x : 0.f) + slope * region[0];
    deriv.y = G.factor[1] * (region[1] == 0 ? grad.y : 0.f) + slope * region[1];
    deriv.z = G.factor[2] * (region[2] == 0 ? grad.z : 0.f) + slope * region[2];
    return f + penalty;
}

// charge map lookup (charge-dependent scoring only), out of line; returns
// (energy, derivative).  Results come back by value so that no caller
// variable has its address taken.
__device__ __noinline__ float4 grid_charge32(int t, float3 loc, float slope, float v) {
    float3 d;
    const float e = grid_aux32(sG32, t, true, loc, slope, v, d);
    return make_float4(e, d.x, d.y, d.z);
}

// table lookup with charge-weighted components (precalculate_linear element
// eval_deriv); out of line, charge-dependent scoring only; returns (e, dor)
__device__ __noinline__ float2 table32_nc(int p, bool swap, float qa, float qb, float r2) {
    const DTables32& T = sT32;
    if (swap) { const float t = qa; qa = qb; qb = t; }
    const float rf = T.factor * r2;
    const int i1 = (int)rf;
    const float rem = rf - (float)i1;
    const float4* b = T.tab + ((size_t)p * T.n + i1) * T.nc;
    const float4 c0 = __ldg(b), c1 = __ldg(b + 1), c2 = __ldg(b + 2), c3 = __ldg(b + 3);
    const float aa = fabsf(qa), bb = fabsf(qb), ab = qa * qb;
    const float e1 = c0.x + aa * c1.x + bb * c2.x + ab * c3.x, e2 = c0.z + aa * c1.z + bb * c2.z + ab * c3.z;
    const float d1 = c0.y + aa * c1.y + bb * c2.y + ab * c3.y, d2 = c0.w + aa * c1.w + bb * c2.w + ab * c3.w;
    return make_float2(e1 + rem * (e2 - e1), d1 + rem * (d2 - d1));
}

// ---- chain teams ------------------------------------------------------------------------------
// A chain may run on a team of G warps (G = 1, 2, 4; the reference's
// threads_per_chain 32, 64, 128), for latency when the device has warps to
// spare.  The team's first warp, the leader, runs the chain: mutation,
// BFGS, line searches, model::set and the derivative.  At every evaluation
// it hands the grid and pair terms out: warp k of the team takes atoms
// k, k + G, ... and a contiguous share of the pair chunks, adding forces
// into its own workspace's force array.  The leader then sums the G
// energies and force arrays in team order, so a team's results do not
// depend on scheduling (they differ from one warp's only by the order of
// FP32 additions).  The hand-out is two named-barrier phases per
// evaluation (barrier id: team index + 1, 32 G threads); helpers take their
// command (the caps, slope and an opcode) from their own workspace's
// scratch words, which the leader writes before the first phase.
constexpr unsigned kTeamEval = 1u, kTeamExit = 2u;
// scratch words of a helper warp's workspace: [0, 4) caps v and slope,
// [4] opcode; [8] energy share, [9] grid lookups, [10] pair lookups
constexpr int kTeamOp = 4, kTeamE = 8, kTeamGrid = 9, kTeamPairs = 10;

template <int G>
__device__ __forceinline__ void team_bar() {
    static_assert(G == 2 || G == 4, "teams of 2 or 4 warps");
    // immediate barrier ids, so that a kernel reserves only the ones it uses
    const int t = (int)(threadIdx.x >> 5) / G;  // the team's index in its block (at most 8 warps)
    if (G == 4) {
        if (t == 0) asm volatile("bar.sync 1, 128;" ::: "memory");
        else asm volatile("bar.sync 2, 128;" ::: "memory");
    } else {
        if (t == 0) asm volatile("bar.sync 1, 64;" ::: "memory");
        else if (t == 1) asm volatile("bar.sync 2, 64;" ::: "memory");
        else if (t == 2) asm volatile("bar.sync 3, 64;" ::: "memory");
        else asm volatile("bar.sync 4, 64;" ::: "memory");
    }
}
// leader: the command for every helper of its team, then the first phase
template <int G>
__device__ __forceinline__ void team_publish(const W32& w, float3 v, float slope, unsigned op) {
    if (w.lane > 0 && w.lane < G) {
        unsigned* S = sp<unsigned>(w.ws + w.lane * sWsStride + smodel().L.scratch);
        S[0] = __float_as_uint(v.x);
        S[1] = __float_as_uint(v.y);
        S[2] = __float_as_uint(v.z);
        S[3] = __float_as_uint(slope);
        S[kTeamOp] = op;
    }
    team_bar<G>();
}

// The grid and pair terms of model::eval_deriv for warp k of a team of G
// (G = 1: the whole of them).  X: the chain's coordinates; F: this warp's
// force array (every movable atom's entry is written).  Returns the warp's
// energy share (same on every lane); adds its lookups to ghits and hits.
template <int G>
__device__ __forceinline__ float eval_terms32(const W32& w, int k, const float4* X, float4* F, float3 v, float slope,
                                              unsigned& ghits, unsigned& hits) {
    const SModel& m = smodel();
    SG_T0(t_grid);
    float e = 0;
    // grid part; every movable atom gets its force reset (hydrogens: zero)
    const int nmov = m.nmov;
    const int* TYPE = sp<const int>(m.type);
    const float4* LQ = sp<const float4>(m.local32);
    if (G > 1) {  // the atoms of other warps start at zero in this warp's array
        for (int i = w.lane; i < nmov; i += 32) F[i] = make_float4(0, 0, 0, 0);
        __syncwarp();
    }
    for (int i = w.lane * G + k; i < nmov; i += 32 * G) {
        const int t = TYPE[i];
        float3 d = make_float3(0, 0, 0);
        if (t < kNumTypes && !is_h(t)) {
            const float3 loc = f3(X[i]);
            e += grid_aux32(sG32, t, false, loc, slope, v.y, d);
            ghits++;
            const float q = LQ[i].w;
            if (q != 0.f && sG32.c32[t]) {
                const float4 cd = grid_charge32(t, loc, slope, v.y);
                e += q * cd.x;
                d = d + q * make_float3(cd.y, cd.z, cd.w);
                ghits++;
            }
        }
        F[i] = make_float4(d.x, d.y, d.z, 0);
    }
    __syncwarp();
    SG_T1(t_grid, 1);
    SG_T0(t_pairs);
    // Pairs: intramolecular (v[0]) and other (v[2]), SG_PAIR_CHUNKS chunks
    // of 32 in flight.  Within a chunk no atom is twice a first atom or twice a
    // second atom, so the force updates are plain read-add-writes: first
    // atoms, sync, second atoms, sync.  This warp's chunks: [c0, c1).
    const int nch = m.npchunks;
    const int c0 = k * nch / G, c1 = (k + 1) * nch / G;
    const uint32_t* PS = sp<const uint32_t>(m.pslot);
    const DTables32 T = sT32;
    const int lane = w.lane;
    uint32_t nsl[SG_PAIR_CHUNKS];  // next round's slots, loaded a round ahead
#pragma unroll
    for (int u = 0; u < SG_PAIR_CHUNKS; u++) nsl[u] = c0 + u < c1 ? PS[(c0 + u) * 32 + lane] : kSlotEmpty;
    for (int c = c0; c < c1; c += SG_PAIR_CHUNKS) {
        const int live = min(SG_PAIR_CHUNKS, c1 - c);  // chunks this round (warp-uniform)
        uint32_t sl[SG_PAIR_CHUNKS];
        int ia[SG_PAIR_CHUNKS], ib[SG_PAIR_CHUNKS];
        float3 r[SG_PAIR_CHUNKS];
        float r2[SG_PAIR_CHUNKS];
        bool ok[SG_PAIR_CHUNKS];
#pragma unroll
        for (int u = 0; u < SG_PAIR_CHUNKS; u++) {
            sl[u] = nsl[u];
            nsl[u] = c + SG_PAIR_CHUNKS + u < c1 ? PS[(c + SG_PAIR_CHUNKS + u) * 32 + lane] : kSlotEmpty;
            ia[u] = sl[u] & 0xff;
            ib[u] = (sl[u] >> 8) & 0xff;
            r[u] = f3(X[ib[u]]) - f3(X[ia[u]]);
            r2[u] = dot3(r[u], r[u]);
            ok[u] = ((sl[u] >> 16) & kSlotPairMask) != kSlotPairMask && r2[u] < T.cutoff_sqr;
        }
        float4 tv[SG_PAIR_CHUNKS];
        float rem[SG_PAIR_CHUNKS];
        if (T.nc == 1) {  // issue every table load before using any
#pragma unroll
            for (int u = 0; u < SG_PAIR_CHUNKS; u++) {
                const float rf = T.factor * r2[u];
                const int i1 = ok[u] ? (int)rf : 0;
                rem[u] = rf - (float)i1;
                tv[u] = ok[u] ? __ldg(T.tab + (int)(((sl[u] >> 16) & 0x1ffu) * (unsigned)T.n + (unsigned)i1)) : make_float4(0, 0, 0, 0);
            }
        }
        float3 f[SG_PAIR_CHUNKS];
#pragma unroll
        for (int u = 0; u < SG_PAIR_CHUNKS; u++) {
            f[u] = make_float3(0, 0, 0);
            if (!ok[u]) continue;
            float pe, dor;
            if (T.nc == 1) {
                pe = tv[u].x + rem[u] * (tv[u].z - tv[u].x);
                dor = tv[u].y + rem[u] * (tv[u].w - tv[u].y);
            } else {
                const float2 ed = table32_nc((sl[u] >> 16) & 0x1ff, (sl[u] & kSlotSwap) != 0, LQ[ia[u]].w, LQ[ib[u]].w, r2[u]);
                pe = ed.x;
                dor = ed.y;
            }
            f[u] = dor * r[u];
            const float vv = (sl[u] & kSlotIntra) ? v.x : v.z;
            if (pe > 0) {
                const float tt = (vv < 1.1920929e-07f) ? 0.f : __fdividef(vv, vv + pe);
                pe *= tt;
                f[u] = (tt * tt) * f[u];
            }
            e += pe;
            hits++;
        }
#pragma unroll
        for (int u = 0; u < SG_PAIR_CHUNKS; u++) {
            if (u >= live) break;
            if (ok[u]) {
                float4 t = F[ia[u]];
                t.x -= f[u].x; t.y -= f[u].y; t.z -= f[u].z;
                F[ia[u]] = t;
            }
            __syncwarp();
            if (ok[u]) {
                float4 t = F[ib[u]];
                t.x += f[u].x; t.y += f[u].y; t.z += f[u].z;
                F[ib[u]] = t;
            }
            __syncwarp();
        }
    }
    e = warp_sum(e);
    __syncwarp();
    SG_T1(t_pairs, 2);
    return e;
}

// a helper warp of a chain team: serves the leader's evaluations until it
// sends kTeamExit
template <int G>
__device__ __noinline__ void team_help32() {
    const W32 w = here();
    const SModel& m = smodel();
    const int k = (int)(threadIdx.x >> 5) % G;
    const float4* X = sp<const float4>(w.ws - k * sWsStride + m.L.coords);  // the leader's coordinates
    unsigned* S = w.counters();
    for (;;) {
        team_bar<G>();  // the leader's command and coordinates are in
        if (S[kTeamOp] != kTeamEval) break;
        const float3 v = make_float3(__uint_as_float(S[0]), __uint_as_float(S[1]), __uint_as_float(S[2]));
        const float slope = __uint_as_float(S[3]);
        unsigned gh = 0, ph = 0;
        const float e = eval_terms32<G>(w, k, X, w.force(), v, slope, gh, ph);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            gh += __shfl_xor_sync(kFull32, gh, o);
            ph += __shfl_xor_sync(kFull32, ph, o);
        }
        if (w.lane == 0) {
            S[kTeamE] = __float_as_uint(e);
            S[kTeamGrid] = gh;
            S[kTeamPairs] = ph;
        }
        team_bar<G>();  // this warp's forces and energy share are in
    }
}

// model::eval_deriv in FP32 on a team of G warps (called by the leader);
// returns the energy (same on every lane), writes g (FP64)
template <int G>
__device__ __noinline__ float eval_deriv32(int conf_at, float3 v, float slope, int g_at) {
    const W32 w = here();
    const SModel& m = smodel();
    double* g = sp<double>(g_at);
    SG_T0(t_set);
    set_conf32(conf_at);
    SG_T1(t_set, 0);
    if constexpr (G > 1) team_publish<G>(w, v, slope, kTeamEval);
    float4* X = w.coords();
    float4* Fz = w.force();
    const int nmov = m.nmov;
    unsigned ghits = 0, hits = 0;
    float e = eval_terms32<G>(w, 0, X, Fz, v, slope, ghits, hits);
    if constexpr (G > 1) {
        team_bar<G>();  // the helpers' shares are in
#pragma unroll
        for (int k = 1; k < G; k++) {
            const unsigned* S = sp<const unsigned>(w.ws + k * sWsStride + m.L.scratch);
            e += __uint_as_float(S[kTeamE]);
            if (w.lane == 0) {
                ghits += S[kTeamGrid];
                hits += S[kTeamPairs];
            }
        }
    }
    SG_T0(t_der);
    // Derivative.  A frame's subtree owns the contiguous atom range
    // [fbegin, fsub_end), so its force and torque are differences of two
    // prefix sums over atoms: F_sub = PF[E] - PF[b], and with
    // c_i = (x_i - o_ref) x F_i, T_sub = PC[E] - PC[b] - (o_f - o_ref) x F_sub.
    // Torques are taken about the first root's origin to keep them small.
    float4* O = w.origin();
    float4* PF = sp<float4>(w.at(m.L.pf));
    float4* PC = sp<float4>(w.at(m.L.pc));
    const float3 oref = f3(O[0]);
    float3 cf = make_float3(0, 0, 0), cc = make_float3(0, 0, 0);
    for (int base = 0; base < nmov; base += 32) {
        const int i = base + w.lane;
        float3 F = make_float3(0, 0, 0), Cq = make_float3(0, 0, 0);
        if (i < nmov) {
            F = f3(Fz[i]);
#pragma unroll
            for (int k = 1; k < G; k++) F = F + f3(sp<const float4>(w.ws + k * sWsStride + m.L.force)[i]);
            Cq = cross3(f3(X[i]) - oref, F);
        }
        float3 iF = F, iC = Cq;
        SG_ROLLED
        for (int off = 1; off < 32; off <<= 1) {
            const float a0 = __shfl_up_sync(kFull32, iF.x, off), a1 = __shfl_up_sync(kFull32, iF.y, off),
                        a2 = __shfl_up_sync(kFull32, iF.z, off), b0 = __shfl_up_sync(kFull32, iC.x, off),
                        b1 = __shfl_up_sync(kFull32, iC.y, off), b2 = __shfl_up_sync(kFull32, iC.z, off);
            if (w.lane >= off) {
                iF = iF + make_float3(a0, a1, a2);
                iC = iC + make_float3(b0, b1, b2);
            }
        }
        if (i < nmov) {  // exclusive prefix at i
            const float3 eF = cf + (iF - F), eC = cc + (iC - Cq);
            PF[i] = make_float4(eF.x, eF.y, eF.z, 0);
            PC[i] = make_float4(eC.x, eC.y, eC.z, 0);
        }
        cf = cf + make_float3(__shfl_sync(kFull32, iF.x, 31), __shfl_sync(kFull32, iF.y, 31), __shfl_sync(kFull32, iF.z, 31));
        cc = cc + make_float3(__shfl_sync(kFull32, iC.x, 31), __shfl_sync(kFull32, iC.y, 31), __shfl_sync(kFull32, iC.z, 31));
    }
    if (w.lane == 0) {
        PF[nmov] = make_float4(cf.x, cf.y, cf.z, 0);
        PC[nmov] = make_float4(cc.x, cc.y, cc.z, 0);
    }
    __syncwarp();
    const int* fbegin = sp<const int>(m.fbegin);
    const int* fsub_end = sp<const int>(m.fsub_end);
    const int* fdof = sp<const int>(m.fdof);
    const int* fkind = sp<const int>(m.fkind);
    for (int f = w.lane; f < m.nframes; f += 32) {
        const int b = fbegin[f], E = fsub_end[f];
        const float3 F = f3(PF[E]) - f3(PF[b]);
        const float3 T = (f3(PC[E]) - f3(PC[b])) - cross3(f3(O[f]) - oref, F);
        const int dof0 = fdof[f];
        if (fkind[f] == SG_FRAME_RIGID) {
            g[dof0] = F.x; g[dof0 + 1] = F.y; g[dof0 + 2] = F.z;
            g[dof0 + 3] = T.x; g[dof0 + 4] = T.y; g[dof0 + 5] = T.z;
        } else {
            g[dof0] = dot3(T, f3(w.axis()[f]));
        }
    }
    __syncwarp();
    SG_T1(t_der, 3);
    unsigned* C = w.counters();
    C[w.lane] += ghits;
    C[32 + w.lane] += hits;
    if (w.lane == 0) C[64] += 1;
    return e;
}

}  // namespace sg
