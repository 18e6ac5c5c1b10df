/* ORACLE — test infrastructure only.
 *
 * CPU restatement, in plain C float arithmetic (no FMA contraction: built with
 * -ffp-contract=off), of the reference's device GAE, rsc::ComputeGAEOnDevice
 * (RocketSimCuda/src/GAECuda.cu:247-300, declared in
 * RocketSimCuda/include/RocketSimCudaTraining.h:17-30):
 *
 *  - the buffer splits at every nonzero terminal into independent segments
 *    [previous terminal + 1, terminal], plus the trailing run after the last terminal
 *    (GAECuda.cu:22-33 marks, :54-69 segment bounds);
 *  - each segment runs the backward recurrence from its end with zero carries
 *    (GAECuda.cu:71-115); a TRUNCATED step bootstraps from
 *    truncValPreds[numTruncs - (truncations before it) - 1], a NORMAL step from 0,
 *    any other step from valPreds[step + 1] (so a non-terminal final step reads
 *    valPreds[T]);
 *  - targetValues = valPreds + advantages (GAECuda.cu:120-129);
 *  - rewClipPortion = (sum |r/std| - sum |clip(r/std)|) / max(sum |r/std|, 1e-7) with
 *    the sums taken per segment and then over segments in buffer order (the reference
 *    adds the per-segment sums with atomics in no fixed order; its own test compares
 *    this value within 1e-4, RocketSimCuda/tests/test_gae_parity.cpp:186-187).
 *
 * For terminals in {0, 1, 2} the result equals the sequential recurrence of the
 * reference's test (test_gae_parity.cpp:24-81); the tests check that on the test's own
 * source compiled from the reference tree.  Nothing in the product links this file.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define GAE_TERM_NORMAL 1
#define GAE_TERM_TRUNCATED 2

/* Returns 0, or -1 when a truncated step has no bootstrap value in range. */
int gae_oracle(const float* rews, const int8_t* terminals, const float* valPreds, const float* truncValPreds,
               int numTruncs, float* advantages, float* targetValues, float* returns, float* rewClipPortion,
               int T, float gamma, float lambda, float returnStd, float clipRange)
{
    int status = 0;
    int truncTotalBefore = 0; /* truncations strictly before the current segment's start */
    float totalRew = 0.0f, totalClipped = 0.0f;
    int start = 0;
    while (start < T) {
        int end = start;
        while (end < T - 1 && terminals[end] == 0)
            ++end;
        /* truncations inside [start, end] */
        int truncIn = 0;
        for (int i = start; i <= end; ++i)
            truncIn += terminals[i] == GAE_TERM_TRUNCATED;
        int truncSeen = 0; /* truncations at positions >= step inside the segment */
        float prevAdvantage = 0.0f, prevReturn = 0.0f, segRew = 0.0f, segClipped = 0.0f;
        for (int step = end; step >= start; --step) {
            int8_t terminal = terminals[step];
            float done = terminal == GAE_TERM_NORMAL ? 1.0f : 0.0f;
            float trunc = terminal == GAE_TERM_TRUNCATED ? 1.0f : 0.0f;
            float curReward;
            if (returnStd > 0.0f) {
                curReward = rews[step] / returnStd;
                segRew += fabsf(curReward);
                if (clipRange > 0.0f)
                    curReward = fminf(fmaxf(curReward, -clipRange), clipRange);
                segClipped += fabsf(curReward);
            } else {
                curReward = rews[step];
                segRew += fabsf(curReward);
            }
            float nextValPred;
            if (terminal == GAE_TERM_TRUNCATED) {
                ++truncSeen;
                int before = truncTotalBefore + truncIn - truncSeen;
                int idx = numTruncs - before - 1;
                if (idx < 0 || idx >= numTruncs) {
                    status = -1;
                    nextValPred = 0.0f;
                } else {
                    nextValPred = truncValPreds[idx];
                }
            } else if (terminal == GAE_TERM_NORMAL) {
                nextValPred = 0.0f;
            } else {
                nextValPred = valPreds[step + 1];
            }
            float predReturn = curReward + gamma * nextValPred * (1.0f - done);
            float delta = predReturn - valPreds[step];
            float notDoneNotTrunc = (1.0f - done) * (1.0f - trunc);
            float curReturn = rews[step] + prevReturn * gamma * notDoneNotTrunc;
            returns[step] = curReturn;
            prevAdvantage = delta + gamma * lambda * notDoneNotTrunc * prevAdvantage;
            advantages[step] = prevAdvantage;
            prevReturn = curReturn;
        }
        totalRew += segRew;
        totalClipped += segClipped;
        truncTotalBefore += truncIn;
        start = end + 1;
    }
    for (int i = 0; i < T; ++i)
        targetValues[i] = valPreds[i] + advantages[i];
    *rewClipPortion = (totalRew - totalClipped) / fmaxf(totalRew, 1e-7f);
    return status;
}
