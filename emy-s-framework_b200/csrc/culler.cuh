// Learned arena-distance culler.
//
// A 3 -> 64 -> 64 -> 1 ReLU MLP maps a point (uu) to an estimate of its distance to the
// soccar arena meshes (the 16 collision meshes; the four static planes are handled by
// their exact distances).  Weights are stored as BF16 and every product is accumulated in
// FP32.  Before each rsb_step launch, cullKernel evaluates the MLP at every body's centre
// and marks the bodies whose whole static-collision reach for the launch is clear:
//
//     min(mlp(p) - margin, exact plane distances(p)) >= reach(body) + vmax * ticks * dt
//
// where reach covers the body's collision shape (the car's box and its four wheel rays)
// plus the contact-breaking threshold, and vmax bounds the body's speed.  The step kernel
// then skips the static tests of marked bodies (wheel rays against meshes and planes, and
// the mesh / plane narrowphase), which cannot find anything while the bound holds.
// The margin is calibrated so that the bound holds on every held-out training point; the
// exact tests stay the fallback for every unmarked body, and in audit mode they also run
// for marked bodies, count every contact or ray hit the bound would have skipped, and
// switch the arena back to the exact path for good.
//
// Training uses the kernels below: exact point-to-mesh distances (brute force over the
// 8,020 triangles), a fused forward + backward pass per 256-point tile with the parameter
// gradients reduced in shared memory, and Adam on FP32 master weights.
#pragma once
#include <cuda_bf16.h>

#include "phys/state.h"

namespace rsb {

constexpr int CM_H = 64;
// flat parameter layout: W1[64][3], b1[64], W2[64][64] (row j = output unit), b2[64], W3[64], b3
constexpr int CP_W1 = 0, CP_B1 = 192, CP_W2 = 256, CP_B2 = 256 + 4096, CP_W3 = CP_B2 + 64, CP_B3 = CP_W3 + 64;
constexpr int CM_NPARAM = CP_B3 + 1;  // 4481
// input / output scaling: inputs are divided by the arena extents, the output is in km
constexpr float CM_SX = 1.f / 4096.f, CM_SY = 1.f / 5120.f, CM_SZ = 1.f / 2048.f, CM_OUT = 1000.f;

// ------------------------------------------------------------------ exact distances

// Closest point on triangle abc to p (the Voronoi-region walk of Ericson, Real-Time
// Collision Detection 5.1.5), returned as the squared distance.
RSB_HD float pointTriDist2(float px, float py, float pz, const float* t) {
    const float ax = t[0], ay = t[1], az = t[2], bx = t[3], by = t[4], bz = t[5], cx = t[6], cy = t[7], cz = t[8];
    const float abx = bx - ax, aby = by - ay, abz = bz - az, acx = cx - ax, acy = cy - ay, acz = cz - az;
    const float apx = px - ax, apy = py - ay, apz = pz - az;
    float qx, qy, qz;
    const float d1 = abx * apx + aby * apy + abz * apz, d2 = acx * apx + acy * apy + acz * apz;
    if (d1 <= 0.f && d2 <= 0.f) {
        qx = ax; qy = ay; qz = az;
    } else {
        const float bpx = px - bx, bpy = py - by, bpz = pz - bz;
        const float d3 = abx * bpx + aby * bpy + abz * bpz, d4 = acx * bpx + acy * bpy + acz * bpz;
        if (d3 >= 0.f && d4 <= d3) {
            qx = bx; qy = by; qz = bz;
        } else {
            const float vc = d1 * d4 - d3 * d2;
            if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
                const float v = d1 / (d1 - d3);
                qx = ax + v * abx; qy = ay + v * aby; qz = az + v * abz;
            } else {
                const float cpx = px - cx, cpy = py - cy, cpz = pz - cz;
                const float d5 = abx * cpx + aby * cpy + abz * cpz, d6 = acx * cpx + acy * cpy + acz * cpz;
                if (d6 >= 0.f && d5 <= d6) {
                    qx = cx; qy = cy; qz = cz;
                } else {
                    const float vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
                        const float w = d2 / (d2 - d6);
                        qx = ax + w * acx; qy = ay + w * acy; qz = az + w * acz;
                    } else {
                        const float va = d3 * d6 - d5 * d4;
                        if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
                            const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
                            qx = bx + w * (cx - bx); qy = by + w * (cy - by); qz = bz + w * (cz - bz);
                        } else {
                            const float den = 1.f / (va + vb + vc);
                            const float v = vb * den, w = vc * den;
                            qx = ax + abx * v + acx * w; qy = ay + aby * v + acy * w; qz = az + abz * v + acz * w;
                        }
                    }
                }
            }
        }
    }
    const float dx = px - qx, dy = py - qy, dz = pz - qz;
    return dx * dx + dy * dy + dz * dz;
}

// Distance (uu) from each point to the nearest of `ntri` triangles (9 floats each, uu).
// Triangles are staged through shared memory in tiles.
constexpr int DIST_TILE = 256;
__global__ void __launch_bounds__(256) meshDistanceKernel(const float* __restrict__ pts, int n,
                                                           const float* __restrict__ tris, int ntri,
                                                           float* __restrict__ out) {
    __shared__ float tile[DIST_TILE * 9];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const float px = live ? pts[3 * i] : 0.f, py = live ? pts[3 * i + 1] : 0.f, pz = live ? pts[3 * i + 2] : 0.f;
    float best = 3.0e38f;
    for (int t0 = 0; t0 < ntri; t0 += DIST_TILE) {
        const int cnt = min(DIST_TILE, ntri - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < cnt * 9; k += blockDim.x) tile[k] = tris[(size_t)t0 * 9 + k];
        __syncthreads();
        for (int t = 0; t < cnt; t++) best = fminf(best, pointTriDist2(px, py, pz, tile + 9 * t));
    }
    if (live) out[i] = sqrtf(best);
}

// ------------------------------------------------------------------ MLP evaluation

// Forward pass with the weights given as floats (already rounded to BF16), in km.
__device__ __forceinline__ float mlpEval(const float* __restrict__ w, float x, float y, float z) {
    const float ix = x * CM_SX, iy = y * CM_SY, iz = z * CM_SZ;
    float h1[CM_H];
#pragma unroll
    for (int i = 0; i < CM_H; i++)
        h1[i] = fmaxf(0.f, fmaf(w[CP_W1 + 3 * i + 2], iz, fmaf(w[CP_W1 + 3 * i + 1], iy, fmaf(w[CP_W1 + 3 * i], ix, w[CP_B1 + i]))));
    float out = w[CP_B3];
    for (int j = 0; j < CM_H; j++) {
        float acc = w[CP_B2 + j];
#pragma unroll
        for (int i = 0; i < CM_H; i++) acc = fmaf(w[CP_W2 + CM_H * j + i], h1[i], acc);
        out = fmaf(w[CP_W3 + j], fmaxf(acc, 0.f), out);
    }
    return out;
}

__device__ __forceinline__ void loadWeights(float* sw, const __nv_bfloat16* __restrict__ wbf) {
    for (int k = threadIdx.x; k < CM_NPARAM; k += blockDim.x) sw[k] = __bfloat162float(wbf[k]);
    __syncthreads();
}

// Predicted distance (uu, before the margin) at each point.
__global__ void mlpPredictKernel(const __nv_bfloat16* __restrict__ wbf, const float* __restrict__ pts, int n,
                                 float* __restrict__ out) {
    __shared__ float sw[CM_NPARAM];
    loadWeights(sw, wbf);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = mlpEval(sw, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]) * CM_OUT;
}

// ------------------------------------------------------------------ training

constexpr int TR_TILE = 256;
constexpr int TR_LD = CM_H + 1;  // padded row of the per-point activations
constexpr size_t TR_SMEM = sizeof(float) * ((size_t)CM_NPARAM + 3 * TR_TILE * TR_LD + TR_TILE * 4);

// Loss over the batch: mean of w * (y - t)^2 with y, t in km and w = overWeight when the
// prediction exceeds the target (over-estimates widen the calibrated margin).
// One block = one tile of TR_TILE points: forward, backward, and the tile's parameter
// gradients reduced in shared memory, then added to `grad` (one atomic per parameter).
__global__ void __launch_bounds__(TR_TILE) mlpTrainKernel(const __nv_bfloat16* __restrict__ wbf,
                                                          const float* __restrict__ pts,
                                                          const float* __restrict__ target, int n, float invBatch,
                                                          float overWeight, float* __restrict__ grad,
                                                          float* __restrict__ lossSum) {
    extern __shared__ float smem[];
    float* sw = smem;                             // weights
    float* H1 = sw + CM_NPARAM;                   // [TR_TILE][TR_LD] layer-1 activations
    float* Z2 = H1 + TR_TILE * TR_LD;             // layer-2 pre-activations, later delta1
    float* D2 = Z2 + TR_TILE * TR_LD;             // layer-2 deltas
    float* X = D2 + TR_TILE * TR_LD;              // [TR_TILE][3] scaled inputs
    float* G = X + TR_TILE * 3;                   // [TR_TILE] dLoss/dy
    loadWeights(sw, wbf);
    const int t = threadIdx.x;
    const int i = blockIdx.x * TR_TILE + t;
    const bool live = i < n;
    const float ix = live ? pts[3 * i] * CM_SX : 0.f, iy = live ? pts[3 * i + 1] * CM_SY : 0.f,
                iz = live ? pts[3 * i + 2] * CM_SZ : 0.f;
    X[3 * t] = ix; X[3 * t + 1] = iy; X[3 * t + 2] = iz;
    float h1[CM_H];
#pragma unroll
    for (int k = 0; k < CM_H; k++) {
        h1[k] = fmaxf(0.f, fmaf(sw[CP_W1 + 3 * k + 2], iz, fmaf(sw[CP_W1 + 3 * k + 1], iy, fmaf(sw[CP_W1 + 3 * k], ix, sw[CP_B1 + k]))));
        H1[t * TR_LD + k] = h1[k];
    }
    float y = sw[CP_B3];
    for (int j = 0; j < CM_H; j++) {
        float acc = sw[CP_B2 + j];
#pragma unroll
        for (int k = 0; k < CM_H; k++) acc = fmaf(sw[CP_W2 + CM_H * j + k], h1[k], acc);
        Z2[t * TR_LD + j] = acc;
        y = fmaf(sw[CP_W3 + j], fmaxf(acc, 0.f), y);
    }
    float g = 0.f, l = 0.f;
    if (live) {
        const float tk = target[i] * (1.f / CM_OUT);
        const float d = y - tk, w = d > 0.f ? overWeight : 1.f;
        g = 2.f * w * d * invBatch;
        l = w * d * d * invBatch;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((t & 31) == 0) atomicAdd(lossSum, l);
    G[t] = g;
    __syncthreads();
    // layer 3
    if (t < CM_H) {
        float s = 0.f;
        for (int p = 0; p < TR_TILE; p++) s = fmaf(G[p], fmaxf(Z2[p * TR_LD + t], 0.f), s);
        atomicAdd(&grad[CP_W3 + t], s);
    } else if (t == CM_H) {
        float s = 0.f;
        for (int p = 0; p < TR_TILE; p++) s += G[p];
        atomicAdd(&grad[CP_B3], s);
    }
    for (int j = 0; j < CM_H; j++) D2[t * TR_LD + j] = Z2[t * TR_LD + j] > 0.f ? g * sw[CP_W3 + j] : 0.f;
    __syncthreads();
    // layer 2: dW2[j][k] = sum_p D2[p][j] * H1[p][k]
    for (int e = t; e < CM_H * CM_H; e += TR_TILE) {
        const int j = e / CM_H, k = e % CM_H;
        float s = 0.f;
        for (int p = 0; p < TR_TILE; p++) s = fmaf(D2[p * TR_LD + j], H1[p * TR_LD + k], s);
        atomicAdd(&grad[CP_W2 + e], s);
    }
    if (t < CM_H) {
        float s = 0.f;
        for (int p = 0; p < TR_TILE; p++) s += D2[p * TR_LD + t];
        atomicAdd(&grad[CP_B2 + t], s);
    }
    // delta1 of this thread's point, written over its Z2 row
    {
        float d1[CM_H];
#pragma unroll
        for (int k = 0; k < CM_H; k++) d1[k] = 0.f;
        for (int j = 0; j < CM_H; j++) {
            const float dj = D2[t * TR_LD + j];
#pragma unroll
            for (int k = 0; k < CM_H; k++) d1[k] = fmaf(dj, sw[CP_W2 + CM_H * j + k], d1[k]);
        }
        __syncthreads();  // every thread is done reading Z2 for layer 3
#pragma unroll
        for (int k = 0; k < CM_H; k++) Z2[t * TR_LD + k] = h1[k] > 0.f ? d1[k] : 0.f;
    }
    __syncthreads();
    // layer 1
    if (t < 3 * CM_H) {
        const int k = t / 3, c = t % 3;
        float s = 0.f;
        for (int p = 0; p < TR_TILE; p++) s = fmaf(Z2[p * TR_LD + k], X[3 * p + c], s);
        atomicAdd(&grad[CP_W1 + t], s);
    } else {
        const int k = t - 3 * CM_H;  // 0..63
        float s = 0.f;
        for (int p = 0; p < TR_TILE; p++) s += Z2[p * TR_LD + k];
        atomicAdd(&grad[CP_B1 + k], s);
    }
}

// Adam on the FP32 master weights; writes the BF16 copy and clears the gradient.
__global__ void adamKernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                           float* __restrict__ grad, __nv_bfloat16* __restrict__ wbf, float lr, float b1, float b2,
                           float c1, float c2, float eps) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= CM_NPARAM) return;
    const float g = grad[k];
    const float mk = b1 * m[k] + (1.f - b1) * g, vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    const float wk = w[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    w[k] = wk;
    wbf[k] = __float2bfloat16_rn(wk);
    grad[k] = 0.f;
}

// ------------------------------------------------------------------ per-launch culling

struct CullParams {
    float margin;        // uu subtracted from the MLP estimate
    float carReach;      // uu: box + wheel rays + contact threshold around the car's centre
    float ballReach;     // uu: radius + contact threshold
    float carVmax, ballVmax;  // uu/s bounds on body speed within a launch
    float dt;
};

// The voxel distance field of the static arena data (ArenaStatic::occDist), Bullet units.
struct VoxelBound {
    const uint16_t* dist;
    V3 mn;
    float inv;
    int X, Y, Z;
    // lower bound (uu) on the distance from a point (uu) to every mesh; 0 off the grid
    RSB_D float at(float x, float y, float z) const {
        const int i = (int)floorf((x * kUuToBt - mn.x) * inv), j = (int)floorf((y * kUuToBt - mn.y) * inv),
                  k = (int)floorf((z * kUuToBt - mn.z) * inv);
        if (i < 0 || j < 0 || k < 0 || i >= X || j >= Y || k >= Z) return 0.f;
        return (float)__ldg(&dist[((size_t)i * Y + j) * Z + k]);
    }
};

// Sets bit b of cull[a] when body b (0 = ball, 1 + s = car s) of arena a cannot reach
// any static geometry during the next `ticks` ticks, by the learned bound (the MLP's estimate
// less the calibrated margin) or, with VOXEL, by the voxel distance field.  Arenas that
// reverted to the exact path (status bit) get no bits.
template <bool VOXEL>
__global__ void cullKernel(const __nv_bfloat16* __restrict__ wbf, VoxelBound vox, CullParams C,
                           const uint32_t* __restrict__ ball, const uint32_t* __restrict__ car,
                           const uint32_t* __restrict__ arena, const int32_t* __restrict__ teamSize, int N, int ticks,
                           uint32_t* __restrict__ cull, int statusWord, uint32_t revertBit) {
    __shared__ float sw[VOXEL ? 1 : CM_NPARAM];
    if (!VOXEL) loadWeights(sw, wbf);
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    uint32_t mask = 0;
    if (!(arena[(size_t)statusWord * N + a] & revertBit)) {
        const int nb = 1 + 2 * teamSize[a];
        const float span = (float)ticks * C.dt;
        for (int b = 0; b < nb; b++) {
            float x, y, z;
            if (b == 0) {
                x = __uint_as_float(ball[(size_t)0 * N + a]) * kBtToUu;
                y = __uint_as_float(ball[(size_t)1 * N + a]) * kBtToUu;
                z = __uint_as_float(ball[(size_t)2 * N + a]) * kBtToUu;
            } else {
                const int s = b - 1;
                x = __uint_as_float(car[((size_t)0 * MAX_CARS + s) * N + a]) * kBtToUu;
                y = __uint_as_float(car[((size_t)1 * MAX_CARS + s) * N + a]) * kBtToUu;
                z = __uint_as_float(car[((size_t)2 * MAX_CARS + s) * N + a]) * kBtToUu;
            }
            const float need = (b == 0 ? C.ballReach + C.ballVmax * span : C.carReach + C.carVmax * span);
            // exact distances to the floor, the ceiling and the two side-wall planes
            const float planes = fminf(fminf(z, ARENA_HEIGHT - z), fminf(x + ARENA_EXTENT_X, ARENA_EXTENT_X - x));
            if (planes < need) continue;
            const float bound = VOXEL ? vox.at(x, y, z) : mlpEval(sw, x, y, z) * CM_OUT - C.margin;
            if (bound >= need) mask |= 1u << b;
        }
    }
    cull[a] = mask;
}

}  // namespace rsb
