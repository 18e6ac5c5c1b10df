// ORACLE PIN — test infrastructure only.
//
// Puts two pieces of the reference's own GAE code behind plain C entry points, compiled
// from the reference tree where it lies (oracle/Makefile, target gae):
//  - gaeref_cpu: the CPU recurrence of the reference's GAE parity test
//    (RocketSimCuda/tests/test_gae_parity.cpp:24-81, `CpuReference`), which this file
//    includes with the test's `main` renamed so that the static function is reachable;
//  - gaeref_device: rsc::ComputeGAEOnDevice (RocketSimCuda/src/GAECuda.cu:247-300),
//    the reference's device GAE, built for sm_100a with --fmad=false as the reference's
//    CMake build does (RocketSimCuda/CMakeLists.txt:116-120).
// The tests use the first to pin the C restatement (gae_oracle.c) and the second to pin
// the engine's kernel to the reference's device results; nothing in the product links it.
#define main rsref_gae_parity_test_main
#include "RocketSimCuda/tests/test_gae_parity.cpp"
#undef main

#include <algorithm>

extern "C" {

int gaeref_cpu(const float* rews, const int8_t* terminals, const float* valPreds, int numValPreds,
               const float* truncValPreds, int numTruncs, int T, float gamma, float lambda, float returnStd,
               float clipRange, float* advantages, float* targetValues, float* returns, float* rewClipPortion)
{
    if (T < 0 || numValPreds < T || numTruncs < 0)
        return -1;
    std::vector<float> r(rews, rews + T), v(valPreds, valPreds + numValPreds), tv(truncValPreds,
                                                                                   truncValPreds + numTruncs);
    std::vector<int8_t> t(terminals, terminals + T);
    CpuGaeOut o = CpuReference(r, t, v, tv, gamma, lambda, returnStd, clipRange);
    std::copy(o.advantages.begin(), o.advantages.end(), advantages);
    std::copy(o.targetValues.begin(), o.targetValues.end(), targetValues);
    std::copy(o.returns.begin(), o.returns.end(), returns);
    *rewClipPortion = o.clipPortion;
    return 0;
}

int gaeref_device(const float* d_rews, const int8_t* d_terminals, const float* d_valPreds,
                  const float* d_truncValPreds, int numTruncs, float* d_advantages, float* d_targetValues,
                  float* d_returns, float* d_rewClipPortion, int T, float gamma, float lambda, float returnStd,
                  float clipRange, void* stream)
{
    rsc::DeviceGAEParams p;
    p.gamma = gamma;
    p.lambda = lambda;
    p.returnStd = returnStd;
    p.clipRange = clipRange;
    rsc::ComputeGAEOnDevice(d_rews, d_terminals, d_valPreds, d_truncValPreds, numTruncs, d_advantages,
                            d_targetValues, d_returns, d_rewClipPortion, T, p, stream);
    return (int)cudaGetLastError();
}

}  // extern "C"
