// GAE over a flat rollout buffer on the device.
//
// Same results, element for element, as the reference's device GAE,
// rsc::ComputeGAEOnDevice (RocketSimCuda/src/GAECuda.cu:247-300): the buffer splits at every
// nonzero terminal into independent segments, each segment runs the backward recurrence of
// GAECuda.cu:71-115 from its end with zero carries, and targetValues = valPreds + advantages
// (GAECuda.cu:120-129).  Compiled with --fmad=false, so each multiply and add rounds as the
// reference's --fmad=false build does.
//
// Layout of the work (three launches, no host round trip):
//   gaeSummaryKernel  one block per 4,096-element chunk: truncations in the chunk and the
//                     position of its last nonzero terminal;
//   gaeScanKernel     one block: exclusive prefix (truncations before each chunk, last
//                     terminal before each chunk);
//   gaeSegmentKernel  one block per chunk: stages the chunk's rewards, values and terminals in
//                     shared memory with coalesced loads, lists the segments that END in the
//                     chunk, runs each one on its own thread (a segment that began in an earlier
//                     chunk walks on into global memory), and writes the chunk's results back
//                     with coalesced stores.  Every element is written by the thread of the
//                     segment that contains it and by no other.  Per-block sums of |r/std| and
//                     |clip(r/std)| go to a scratch row; the last block to finish (a ticket
//                     counter, no waiting) adds them in block order and writes rewClipPortion.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "rsb.h"

namespace rsb {
void setGlobalError(const std::string& msg);
}

namespace {

constexpr int kGaeThreads = 256;
constexpr int kGaePerThread = 16;
constexpr int kGaeChunk = kGaeThreads * kGaePerThread;  // elements per block
constexpr int kPosBits = 13;                             // chunk-relative position field of a segment entry
constexpr int kPosMask = (1 << kPosBits) - 1;
constexpr int8_t kTermNormal = 1;
constexpr int8_t kTermTruncated = 2;
// largest T: chunk arithmetic stays inside int32
constexpr int32_t kGaeMaxT = INT32_MAX - 2 * kGaeChunk;

// Shared memory of gaeSegmentKernel.  The float rows are padded by one word per 32 elements,
// so that lanes walking segments whose lengths are multiples of 32 (one trajectory of a
// 32-step rollout per lane) fall into different banks.
constexpr int kPadded = kGaeChunk + kGaeChunk / 32;
__host__ __device__ constexpr int padIdx(int i) { return i + (i >> 5); }
constexpr size_t kSmemRew = sizeof(float) * kPadded;        // rewards, then advantages
constexpr size_t kSmemRet = sizeof(float) * kPadded;        // returns
constexpr size_t kSmemVal = sizeof(float) * (kPadded + 4);  // values + the one after the chunk
constexpr size_t kSmemSeg = sizeof(int) * (kGaeChunk + 4);  // segment ends
constexpr size_t kSmemTerm = kGaeChunk;                     // terminals (16-byte aligned)
constexpr size_t kSmemSegment = kSmemRew + kSmemRet + kSmemVal + kSmemSeg + kSmemTerm;
static_assert((kSmemRew + kSmemRet + kSmemVal + kSmemSeg) % 16 == 0, "terminal row must be 16-byte aligned");

struct GaeArgs {
    const float* rews;
    const int8_t* term;
    const float* vals;
    const float* truncVals;
    int numTruncs;
    float* adv;
    float* tgt;
    float* ret;
    float* clipPortion;
    int T;
    int nChunks;
    float gamma, lambda, returnStd, clipRange;
    const int2* pre;
    float2* part;
    unsigned* ticket;
};

__device__ __forceinline__ int warpSum(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warpMax(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Truncations and the last nonzero terminal of each chunk.  Thread t reads bytes
// [16 t, 16 t + 16) of its chunk, as one 16-byte load when the row is 16-byte aligned.
template <bool kVec>
__global__ void __launch_bounds__(kGaeThreads) gaeSummaryKernel(const int8_t* __restrict__ term, int T,
                                                                int2* __restrict__ sum) {
    const int base = blockIdx.x * kGaeChunk;
    const int len = min(kGaeChunk, T - base);
    const int j0 = threadIdx.x * kGaePerThread;
    int tr = 0, last = -1;
    if (kVec && j0 + kGaePerThread <= len) {
        const uint4 w = __ldg(reinterpret_cast<const uint4*>(term + base + j0));
        const unsigned words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int k = 0; k < kGaePerThread; ++k) {
            const int8_t t = (int8_t)(words[k >> 2] >> (8 * (k & 3)));
            tr += t == kTermTruncated;
            if (t != 0) last = base + j0 + k;
        }
    } else {
        for (int k = 0; k < kGaePerThread && j0 + k < len; ++k) {
            const int8_t t = __ldg(term + base + j0 + k);
            tr += t == kTermTruncated;
            if (t != 0) last = base + j0 + k;
        }
    }
    tr = warpSum(tr);
    last = warpMax(last);
    __shared__ int sTr[kGaeThreads / 32], sLast[kGaeThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sTr[warp] = tr;
        sLast[warp] = last;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0, m = -1;
        for (int w = 0; w < kGaeThreads / 32; ++w) {
            a += sTr[w];
            m = max(m, sLast[w]);
        }
        sum[blockIdx.x] = make_int2(a, m);
    }
}

// Exclusive prefix over chunks: truncations before the chunk, last terminal before it (-1).
__global__ void __launch_bounds__(1024) gaeScanKernel(const int2* __restrict__ sum, int n, int2* __restrict__ pre) {
    __shared__ int wSum[32], wMax[32];
    __shared__ int carrySum, carryMax;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        carrySum = 0;
        carryMax = -1;
    }
    __syncthreads();
    for (int base = 0; base < n; base += 1024) {
        const int i = base + (int)threadIdx.x;
        const int2 v = i < n ? sum[i] : make_int2(0, -1);
        int s = v.x, m = v.y;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int s2 = __shfl_up_sync(0xffffffffu, s, o);
            const int m2 = __shfl_up_sync(0xffffffffu, m, o);
            if (lane >= o) {
                s += s2;
                m = max(m, m2);
            }
        }
        int exM = __shfl_up_sync(0xffffffffu, m, 1);
        if (lane == 0) exM = -1;
        if (lane == 31) {
            wSum[warp] = s;
            wMax[warp] = m;
        }
        __syncthreads();
        if (warp == 0) {
            int ws = wSum[lane], wm = wMax[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int s2 = __shfl_up_sync(0xffffffffu, ws, o);
                const int m2 = __shfl_up_sync(0xffffffffu, wm, o);
                if (lane >= o) {
                    ws += s2;
                    wm = max(wm, m2);
                }
            }
            wSum[lane] = ws;
            wMax[lane] = wm;
        }
        __syncthreads();
        const int addS = carrySum + (warp ? wSum[warp - 1] : 0);
        const int addM = max(carryMax, warp ? wMax[warp - 1] : -1);
        if (i < n) pre[i] = make_int2(addS + s - v.x, max(addM, exM));
        __syncthreads();
        if (threadIdx.x == 1023) {
            carrySum = addS + s;
            carryMax = max(addM, m);
        }
        __syncthreads();
    }
}

// One backward step of GAECuda.cu:77-113 (the same operations in the same order).
struct GaeCarry {
    float adv, ret, rew, clipped;
};

__device__ __forceinline__ void gaeStep(const GaeArgs& a, float rew, int8_t terminal, float val, float nextVal,
                                        int truncBefore, GaeCarry& c, float& advOut, float& retOut) {
    const float done = terminal == kTermNormal ? 1.0f : 0.0f;
    const float trunc = terminal == kTermTruncated ? 1.0f : 0.0f;
    float curReward;
    if (a.returnStd > 0.0f) {
        curReward = rew / a.returnStd;
        c.rew += fabsf(curReward);
        if (a.clipRange > 0.0f) curReward = fminf(fmaxf(curReward, -a.clipRange), a.clipRange);
        c.clipped += fabsf(curReward);
    } else {
        curReward = rew;
        c.rew += fabsf(curReward);
    }
    float nextValPred;
    if (terminal == kTermTruncated) {
        const int idx = a.numTruncs - truncBefore - 1;
        // a count that does not match the truncated steps reads nothing out of range
        nextValPred = (idx >= 0 && idx < a.numTruncs) ? __ldg(a.truncVals + idx) : 0.0f;
    } else if (terminal == kTermNormal) {
        nextValPred = 0.0f;
    } else {
        nextValPred = nextVal;
    }
    const float predReturn = curReward + a.gamma * nextValPred * (1.0f - done);
    const float delta = predReturn - val;
    const float notDoneNotTrunc = (1.0f - done) * (1.0f - trunc);
    const float curReturn = rew + c.ret * a.gamma * notDoneNotTrunc;
    retOut = curReturn;
    c.adv = delta + a.gamma * a.lambda * notDoneNotTrunc * c.adv;
    advOut = c.adv;
    c.ret = curReturn;
}

// The same step for a running element (terminal 0), the only kind a segment holds before its
// end: done = trunc = 0 make the reference's factors (1 - done) and (1 - done)(1 - trunc)
// exactly 1, and multiplying by 1 changes no finite value, so the products are dropped.
__device__ __forceinline__ void gaeStepRunning(const GaeArgs& a, float rew, float val, float nextVal, GaeCarry& c,
                                               float& advOut, float& retOut) {
    float curReward;
    if (a.returnStd > 0.0f) {
        curReward = rew / a.returnStd;
        c.rew += fabsf(curReward);
        if (a.clipRange > 0.0f) curReward = fminf(fmaxf(curReward, -a.clipRange), a.clipRange);
        c.clipped += fabsf(curReward);
    } else {
        curReward = rew;
        c.rew += fabsf(curReward);
    }
    const float predReturn = curReward + a.gamma * nextVal;
    const float delta = predReturn - val;
    const float curReturn = rew + c.ret * a.gamma;
    retOut = curReturn;
    c.adv = delta + a.gamma * a.lambda * c.adv;
    advOut = c.adv;
    c.ret = curReturn;
}

template <bool kVec>
__global__ void __launch_bounds__(kGaeThreads) gaeSegmentKernel(GaeArgs a) {
    extern __shared__ float4 gaeSmem[];
    float* sRew = reinterpret_cast<float*>(gaeSmem);  // rewards, overwritten by advantages
    float* sRet = sRew + kPadded;
    float* sVal = sRet + kPadded;
    int* sSeg = reinterpret_cast<int*>(sVal + kPadded + 4);
    int8_t* sTerm = reinterpret_cast<int8_t*>(sSeg + kGaeChunk + 4);
    __shared__ int sWarpCount[kGaeThreads / 32];
    __shared__ float2 sWarpSum[kGaeThreads / 32];
    __shared__ int sTotal;
    __shared__ bool sLastBlock;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int base = blockIdx.x * kGaeChunk;
    const int len = min(kGaeChunk, a.T - base);

    // 1. stage the chunk (coalesced; terminals as 4-byte words when aligned)
#pragma unroll
    for (int k = 0; k < kGaePerThread; ++k) {
        const int j = k * kGaeThreads + tid;
        if (j < len) {
            sRew[padIdx(j)] = __ldg(a.rews + base + j);
            sVal[padIdx(j)] = __ldg(a.vals + base + j);
        }
    }
    if (kVec) {
#pragma unroll
        for (int k = 0; k < kGaePerThread / 4; ++k) {
            const int w = k * kGaeThreads + tid;
            if (4 * w + 4 <= len) {
                reinterpret_cast<int*>(sTerm)[w] = __ldg(reinterpret_cast<const int*>(a.term + base) + w);
            } else {
                for (int b = 4 * w; b < len && b < 4 * w + 4; ++b) sTerm[b] = __ldg(a.term + base + b);
            }
        }
    } else {
        for (int j = tid; j < len; j += kGaeThreads) sTerm[j] = __ldg(a.term + base + j);
    }
    if (tid == 0) {
        // the value after the chunk; past the buffer the reference reads valPreds[T] only
        // for a non-terminal final step (GAECuda.cu:101-102)
        const int nxt = base + len;
        float v = 0.0f;
        if (nxt < a.T) v = __ldg(a.vals + nxt);
        else if (__ldg(a.term + a.T - 1) == 0) v = __ldg(a.vals + a.T);
        sVal[padIdx(len)] = v;
    }
    __syncthreads();

    // 2. list the segments that end in this chunk: nonzero terminals, and the buffer's last
    //    element when it is not terminal (the trailing run)
    const bool lastChunk = base + len == a.T;
    const int own0 = tid * kGaePerThread;
    unsigned endMask = 0, truncMask = 0;
    {
        const uint4 w = reinterpret_cast<const uint4*>(sTerm)[tid];  // bytes past len are not read below
        const unsigned words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int k = 0; k < kGaePerThread; ++k) {
            const int j = own0 + k;
            if (j < len) {
                const int8_t t = (int8_t)(words[k >> 2] >> (8 * (k & 3)));
                if (t != 0 || (lastChunk && j == len - 1)) endMask |= 1u << k;
                if (t == kTermTruncated) truncMask |= 1u << k;
            }
        }
    }
    // block exclusive scan of (ends | truncations << 16)
    const int packed = __popc(endMask) | (__popc(truncMask) << 16);
    int incl = packed;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) sWarpCount[warp] = incl;
    __syncthreads();
    if (tid == 0) {
        int run = 0;
        for (int w = 0; w < kGaeThreads / 32; ++w) {
            const int c = sWarpCount[w];
            sWarpCount[w] = run;
            run += c;
        }
        sTotal = run;
    }
    __syncthreads();
    {
        const int ex = incl - packed + sWarpCount[warp];
        int idx = ex & 0xffff;
        int trb = ex >> 16;
#pragma unroll
        for (int k = 0; k < kGaePerThread; ++k) {
            if (endMask >> k & 1u) sSeg[idx++] = (own0 + k) | (trb << kPosBits);
            if (truncMask >> k & 1u) ++trb;
        }
    }
    __syncthreads();
    const int nSeg = sTotal & 0xffff;
    const int2 pre = a.pre[blockIdx.x];

    // 3. one thread per segment, backward from its end
    float accRew = 0.0f, accClipped = 0.0f;
    for (int s = tid; s < nSeg; s += kGaeThreads) {
        const int e = sSeg[s];
        const int endRel = e & kPosMask;
        const int truncBefore = pre.x + (e >> kPosBits);
        const int start = s == 0 ? pre.y + 1 : base + (sSeg[s - 1] & kPosMask) + 1;
        const int stopRel = max(start - base, 0);
        GaeCarry c{0.0f, 0.0f, 0.0f, 0.0f};
        float adv, ret;
        // the segment's end carries its terminal
        float nextVal = sVal[padIdx(endRel)];
        gaeStep(a, sRew[padIdx(endRel)], sTerm[endRel], nextVal, sVal[padIdx(endRel + 1)], truncBefore, c, adv, ret);
        sRew[padIdx(endRel)] = adv;
        sRet[padIdx(endRel)] = ret;
        // every earlier step of the segment is running
#pragma unroll 4
        for (int rel = endRel - 1; rel >= stopRel; --rel) {
            const float val = sVal[padIdx(rel)];
            gaeStepRunning(a, sRew[padIdx(rel)], val, nextVal, c, adv, ret);
            sRew[padIdx(rel)] = adv;
            sRet[padIdx(rel)] = ret;
            nextVal = val;
        }
        // a segment that began in an earlier chunk continues in global memory
        for (int step = base - 1; step >= start; --step) {
            const float val = __ldg(a.vals + step);
            gaeStepRunning(a, __ldg(a.rews + step), val, nextVal, c, adv, ret);
            a.adv[step] = adv;
            a.ret[step] = ret;
            a.tgt[step] = val + adv;
            nextVal = val;
        }
        accRew += c.rew;
        accClipped += c.clipped;
    }
    __syncthreads();

    // 4. write back the elements of the segments that end here (coalesced)
    const int owned = nSeg > 0 ? (sSeg[nSeg - 1] & kPosMask) + 1 : 0;
#pragma unroll
    for (int k = 0; k < kGaePerThread; ++k) {
        const int j = k * kGaeThreads + tid;
        if (j < owned) {
            const float adv = sRew[padIdx(j)];
            a.adv[base + j] = adv;
            a.ret[base + j] = sRet[padIdx(j)];
            a.tgt[base + j] = sVal[padIdx(j)] + adv;
        }
    }

    // 5. clip-portion sums: block partial, then the last block adds the partials in order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        accRew += __shfl_xor_sync(0xffffffffu, accRew, o);
        accClipped += __shfl_xor_sync(0xffffffffu, accClipped, o);
    }
    if (lane == 0) sWarpSum[warp] = make_float2(accRew, accClipped);
    __syncthreads();
    if (tid == 0) {
        float r = 0.0f, cl = 0.0f;
        for (int w = 0; w < kGaeThreads / 32; ++w) {
            r += sWarpSum[w].x;
            cl += sWarpSum[w].y;
        }
        a.part[blockIdx.x] = make_float2(r, cl);
        __threadfence();
        sLastBlock = atomicAdd(a.ticket, 1u) == (unsigned)(a.nChunks - 1);
    }
    __syncthreads();
    if (!sLastBlock) return;
    __threadfence();
    float r = 0.0f, cl = 0.0f;
    for (int i = tid; i < a.nChunks; i += kGaeThreads) {
        const float2 p = __ldcg(a.part + i);
        r += p.x;
        cl += p.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r += __shfl_xor_sync(0xffffffffu, r, o);
        cl += __shfl_xor_sync(0xffffffffu, cl, o);
    }
    __syncthreads();
    if (lane == 0) sWarpSum[warp] = make_float2(r, cl);
    __syncthreads();
    if (tid == 0) {
        float tr = 0.0f, tc = 0.0f;
        for (int w = 0; w < kGaeThreads / 32; ++w) {
            tr += sWarpSum[w].x;
            tc += sWarpSum[w].y;
        }
        *a.clipPortion = (tr - tc) / fmaxf(tr, 1e-7f);
    }
}

// Per-device scratch, grown on demand (chunk rows + the ticket).
struct GaeScratch {
    int capacity = 0;
    int2* sum = nullptr;
    int2* pre = nullptr;
    float2* part = nullptr;
    unsigned* ticket = nullptr;
    bool smemSet = false;
};

std::mutex g_gaeMu;
std::vector<GaeScratch> g_gaeScratch;

// Host-buffer staging for rsb_compute_gae_host, per device.
struct GaeHostStage {
    size_t capT = 0, capTrunc = 0;
    float *rews = nullptr, *vals = nullptr, *trunc = nullptr, *adv = nullptr, *tgt = nullptr, *ret = nullptr,
          *clip = nullptr;
    int8_t* term = nullptr;
    cudaStream_t stream = nullptr;
};
std::vector<GaeHostStage> g_gaeHost;

rsb_status ensureScratch(int dev, int nChunks, GaeScratch*& out) {
    if ((int)g_gaeScratch.size() <= dev) g_gaeScratch.resize(dev + 1);
    GaeScratch& s = g_gaeScratch[dev];
    if (!s.smemSet) {
        if (cudaFuncSetAttribute(gaeSegmentKernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmemSegment) != cudaSuccess ||
            cudaFuncSetAttribute(gaeSegmentKernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmemSegment) != cudaSuccess)
            return RSB_ERR_CUDA;
        s.smemSet = true;
    }
    if (s.capacity < nChunks) {
        // the old rows may still be read by work queued earlier on any stream
        if (s.capacity > 0 && cudaDeviceSynchronize() != cudaSuccess) return RSB_ERR_CUDA;
        cudaFree(s.sum);
        cudaFree(s.pre);
        cudaFree(s.part);
        if (!s.ticket && cudaMalloc(&s.ticket, sizeof(unsigned)) != cudaSuccess) return RSB_ERR_NOMEM;
        const int cap = nChunks < 64 ? 64 : nChunks;
        s.capacity = 0;
        s.sum = nullptr;
        s.pre = nullptr;
        s.part = nullptr;
        if (cudaMalloc(&s.sum, sizeof(int2) * cap) != cudaSuccess ||
            cudaMalloc(&s.pre, sizeof(int2) * cap) != cudaSuccess ||
            cudaMalloc(&s.part, sizeof(float2) * cap) != cudaSuccess)
            return RSB_ERR_NOMEM;
        s.capacity = cap;
    }
    out = &s;
    return RSB_OK;
}

rsb_status launchGae(const float* rews, const int8_t* terminals, const float* valPreds, const float* truncValPreds,
                     int32_t numTruncs, float* advantages, float* targetValues, float* returns,
                     float* rewClipPortion, int32_t T, const rsb_gae_params& p, cudaStream_t st) {
    if (T == 0) {
        // no element: the sums are zero, so the portion is 0 / 1e-7 = 0
        return cudaMemsetAsync(rewClipPortion, 0, sizeof(float), st) == cudaSuccess ? RSB_OK : RSB_ERR_CUDA;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return RSB_ERR_CUDA;
    const int nChunks = (T + kGaeChunk - 1) / kGaeChunk;
    GaeScratch* s = nullptr;
    const rsb_status rc = ensureScratch(dev, nChunks, s);
    if (rc != RSB_OK) return rc;
    GaeArgs a;
    a.rews = rews;
    a.term = terminals;
    a.vals = valPreds;
    a.truncVals = truncValPreds;
    a.numTruncs = numTruncs;
    a.adv = advantages;
    a.tgt = targetValues;
    a.ret = returns;
    a.clipPortion = rewClipPortion;
    a.T = T;
    a.nChunks = nChunks;
    a.gamma = p.gamma;
    a.lambda = p.lambda;
    a.returnStd = p.return_std;
    a.clipRange = p.clip_range;
    a.pre = s->pre;
    a.part = s->part;
    a.ticket = s->ticket;
    const bool vec = (reinterpret_cast<uintptr_t>(terminals) & 15) == 0;
    if (vec) gaeSummaryKernel<true><<<nChunks, kGaeThreads, 0, st>>>(terminals, T, s->sum);
    else gaeSummaryKernel<false><<<nChunks, kGaeThreads, 0, st>>>(terminals, T, s->sum);
    gaeScanKernel<<<1, 1024, 0, st>>>(s->sum, nChunks, s->pre);
    if (cudaMemsetAsync(s->ticket, 0, sizeof(unsigned), st) != cudaSuccess) return RSB_ERR_CUDA;
    if (vec) gaeSegmentKernel<true><<<nChunks, kGaeThreads, kSmemSegment, st>>>(a);
    else gaeSegmentKernel<false><<<nChunks, kGaeThreads, kSmemSegment, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? RSB_OK : RSB_ERR_CUDA;
}

bool validArgs(const void* rews, const void* terminals, const void* valPreds, const void* truncValPreds,
               int32_t numTruncs, const void* advantages, const void* targetValues, const void* returns,
               const void* rewClipPortion, int32_t T, const rsb_gae_params* params) {
    if (!params || !rewClipPortion || T < 0 || T > kGaeMaxT || numTruncs < 0) return false;
    if (numTruncs > 0 && !truncValPreds) return false;
    if (T > 0 && (!rews || !terminals || !valPreds || !advantages || !targetValues || !returns)) return false;
    return true;
}

}  // namespace

extern "C" {

rsb_status rsb_gae_default_params(rsb_gae_params* out) {
    if (!out) return RSB_ERR_INVALID;
    out->gamma = 0.99f;
    out->lambda = 0.95f;
    out->return_std = 0.0f;
    out->clip_range = 0.0f;
    return RSB_OK;
}

rsb_status rsb_compute_gae(const float* rews, const int8_t* terminals, const float* val_preds,
                           const float* trunc_val_preds, int32_t num_truncs, float* advantages, float* target_values,
                           float* returns, float* rew_clip_portion, int32_t T, const rsb_gae_params* params,
                           void* stream) {
    std::lock_guard<std::mutex> lock(g_gaeMu);
    if (!validArgs(rews, terminals, val_preds, trunc_val_preds, num_truncs, advantages, target_values, returns,
                   rew_clip_portion, T, params)) {
        rsb::setGlobalError("rsb_compute_gae: invalid argument");
        return RSB_ERR_INVALID;
    }
    const rsb_status rc = launchGae(rews, terminals, val_preds, trunc_val_preds, num_truncs, advantages,
                                    target_values, returns, rew_clip_portion, T, *params,
                                    reinterpret_cast<cudaStream_t>(stream));
    if (rc != RSB_OK) rsb::setGlobalError("rsb_compute_gae: CUDA launch or allocation failed");
    return rc;
}

rsb_status rsb_compute_gae_host(const float* rews, const int8_t* terminals, const float* val_preds,
                                int32_t num_val_preds, const float* trunc_val_preds, int32_t num_truncs,
                                float* advantages, float* target_values, float* returns, float* rew_clip_portion,
                                int32_t T, const rsb_gae_params* params) {
    std::lock_guard<std::mutex> lock(g_gaeMu);
    if (!validArgs(rews, terminals, val_preds, trunc_val_preds, num_truncs, advantages, target_values, returns,
                   rew_clip_portion, T, params) ||
        num_val_preds < T || (T > 0 && terminals[T - 1] == 0 && num_val_preds < T + 1)) {
        rsb::setGlobalError("rsb_compute_gae_host: invalid argument (a non-terminal final step needs T + 1 values)");
        return RSB_ERR_INVALID;
    }
    auto fail = [&](rsb_status rc, const char* what) {
        rsb::setGlobalError(std::string("rsb_compute_gae_host: ") + what);
        return rc;
    };
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(RSB_ERR_CUDA, "no CUDA device");
    if ((int)g_gaeHost.size() <= dev) g_gaeHost.resize(dev + 1);
    GaeHostStage& h = g_gaeHost[dev];
    if (!h.stream && cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(RSB_ERR_CUDA, "stream creation failed");
    const size_t needT = (size_t)T + 1;
    if (h.capT < needT) {
        cudaFree(h.rews);
        cudaFree(h.vals);
        cudaFree(h.adv);
        cudaFree(h.tgt);
        cudaFree(h.ret);
        cudaFree(h.term);
        h.rews = h.vals = h.adv = h.tgt = h.ret = nullptr;
        h.term = nullptr;
        h.capT = 0;
        if (cudaMalloc(&h.rews, needT * 4) != cudaSuccess || cudaMalloc(&h.vals, needT * 4) != cudaSuccess ||
            cudaMalloc(&h.adv, needT * 4) != cudaSuccess || cudaMalloc(&h.tgt, needT * 4) != cudaSuccess ||
            cudaMalloc(&h.ret, needT * 4) != cudaSuccess || cudaMalloc(&h.term, needT) != cudaSuccess)
            return fail(RSB_ERR_NOMEM, "device allocation failed");
        h.capT = needT;
    }
    if (!h.clip && cudaMalloc(&h.clip, sizeof(float)) != cudaSuccess) return fail(RSB_ERR_NOMEM, "allocation failed");
    if (h.capTrunc < (size_t)num_truncs || !h.trunc) {
        cudaFree(h.trunc);
        h.trunc = nullptr;
        const size_t n = num_truncs > 0 ? (size_t)num_truncs : 1;
        if (cudaMalloc(&h.trunc, n * 4) != cudaSuccess) return fail(RSB_ERR_NOMEM, "device allocation failed");
        h.capTrunc = n;
    }
    cudaStream_t st = h.stream;
    const size_t nv = (size_t)(num_val_preds < T + 1 ? num_val_preds : T + 1);
    if (T > 0 && (cudaMemcpyAsync(h.rews, rews, (size_t)T * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
                  cudaMemcpyAsync(h.term, terminals, (size_t)T, cudaMemcpyHostToDevice, st) != cudaSuccess ||
                  cudaMemcpyAsync(h.vals, val_preds, nv * 4, cudaMemcpyHostToDevice, st) != cudaSuccess))
        return fail(RSB_ERR_CUDA, "host to device copy failed");
    if (num_truncs > 0 &&
        cudaMemcpyAsync(h.trunc, trunc_val_preds, (size_t)num_truncs * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return fail(RSB_ERR_CUDA, "host to device copy failed");
    rsb_status rc = launchGae(h.rews, h.term, h.vals, h.trunc, num_truncs, h.adv, h.tgt, h.ret, h.clip, T, *params, st);
    if (rc != RSB_OK) return fail(rc, "launch failed");
    if (T > 0 && (cudaMemcpyAsync(advantages, h.adv, (size_t)T * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                  cudaMemcpyAsync(target_values, h.tgt, (size_t)T * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                  cudaMemcpyAsync(returns, h.ret, (size_t)T * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess))
        return fail(RSB_ERR_CUDA, "device to host copy failed");
    if (cudaMemcpyAsync(rew_clip_portion, h.clip, sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return fail(RSB_ERR_CUDA, "device to host copy failed");
    return cudaStreamSynchronize(st) == cudaSuccess ? RSB_OK : fail(RSB_ERR_CUDA, "stream synchronize failed");
}

}  // extern "C"
