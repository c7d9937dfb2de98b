// ss_narrow.cu -- Bayesian range narrowing from a resident session's average
// strategy, on the device.
//
// The reference narrows a player's range between streets on the host
// (python/hud_solver.py:345-362 feeding python/range_narrowing.py:83-130):
// after a solve it reads the solver player's average strategy at the
// player's first decision node (get_avg_strategy, python/street_solver_gpu.py:
// 497-526: frequencies above 0.001 per action label, keyed by the combo),
// takes P(action | hand) from it, and updates every (c0, c1, w) entry of the
// narrower's range: w' = w * P, or w * 1/max(#distinct P values, 2) for a
// combo the solve did not hold; w' < 0.005 with w > 0 becomes 0.005; then
// all weights are divided by their maximum.  The update is skipped when no
// P is positive.
//
// Here the same steps run in one block on the device, reading the strategy
// sums of the session where the solve left them (no copy of the average
// strategies to the host), in FP64 like the reference's Python floats, so
// the narrowed weights are bit for bit the reference's.
#include "ss_session.h"

#include <cuda_runtime.h>

#include <string>

namespace ssb {

namespace {

constexpr int kNarrowThreads = 1024;
constexpr int kNarrowSort = 2048;     // >= 1326 combos
constexpr double kWeightFloor = 0.005;   // python/range_narrowing.py:47
constexpr double kFreqShown = 0.001;     // python/street_solver_gpu.py:521

__device__ __forceinline__ int combo_id(int a, int b) {   // a < b, 0 .. 1325
    return a * 52 - a * (a + 1) / 2 + (b - a - 1);
}

// One block.  fe / na: the node's first edge and actions; mask: the action
// indices carrying the label (the last of them with a shown frequency wins,
// as in the label dictionary); cards [n][2], w [n] in / out.
__global__ void __launch_bounds__(kNarrowThreads) k_narrow(DevCtx c, int player, int fe, int na, unsigned mask,
                                                           const int *__restrict__ cards, double *w, int n,
                                                           int *applied) {
    __shared__ int last[1326];           // last hand index of each combo in the solve's range, -1 if none
    __shared__ double prob[1326];        // P(action | combo) of the label dictionary
    __shared__ double srt[kNarrowSort];
    __shared__ double red[kNarrowThreads / 32];
    __shared__ int cnt[kNarrowThreads / 32];
    __shared__ int any_pos;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int H = c.H[player];
    const size_t HS = static_cast<size_t>(c.HS);
    for (int i = tid; i < 1326; i += blockDim.x) last[i] = -1;
    if (tid == 0) any_pos = 0;
    __syncthreads();
    for (int h = tid; h < H; h += blockDim.x) {
        const int code = c.hand_code[player * HS + h];
        const int a = code & 0xff, b = (code >> 8) & 0xff;
        if (a == b || a > 51 || b > 51) continue;
        atomicMax(&last[a < b ? combo_id(a, b) : combo_id(b, a)], h);
    }
    __syncthreads();
    // the average strategy of the hand (float32, as the solve's output), then
    // the label's shown frequency
    for (int k = tid; k < 1326; k += blockDim.x) {
        const int h = last[k];
        double p = 0.0;
        if (h >= 0) {
            float v[SS_MAX_ACTIONS];
            float sum = 0.f;
            for (int a = 0; a < na; ++a) {
                float x = c.S[static_cast<size_t>(fe + a) * HS + h];
                x = x < 0.f ? 0.f : x;
                v[a] = x;
                sum += x;
            }
            const float inv = sum > 0.f ? 1.0f / sum : 1.0f / static_cast<float>(na);
            for (int a = 0; a < na; ++a) {
                if (!((mask >> a) & 1u)) continue;
                const double f = static_cast<double>(sum > 0.f ? v[a] * inv : inv);
                if (f > kFreqShown) p = f;
            }
            if (p > 0.0) any_pos = 1;
        }
        prob[k] = p;
    }
    // distinct P values of the dictionary: sort, then count value changes
    for (int i = tid; i < kNarrowSort; i += blockDim.x) srt[i] = (i < 1326 && last[i] >= 0) ? prob[i] : 2.0;
    __syncthreads();
    for (int size = 2; size <= kNarrowSort; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = tid; i < kNarrowSort; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const double x = srt[i], y = srt[j];
                    if ((x > y) == up) {
                        srt[i] = y;
                        srt[j] = x;
                    }
                }
            }
            __syncthreads();
        }
    int local = 0;
    for (int i = tid; i < kNarrowSort; i += blockDim.x)
        if (srt[i] <= 1.5 && (i == 0 || srt[i] != srt[i - 1])) ++local;
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if (lane == 0) cnt[warp] = local;
    __syncthreads();
    if (!any_pos) {
        if (tid == 0) *applied = 0;
        return;
    }
    int distinct = 0;
    for (int i = 0; i < kNarrowThreads / 32; ++i) distinct += cnt[i];
    const double uniform = 1.0 / static_cast<double>(distinct > 2 ? distinct : 2);
    // Bayes update with the floor, then the maximum
    double mx = -1.0;
    for (int i = tid; i < n; i += blockDim.x) {
        const int a = cards[2 * i], b = cards[2 * i + 1];
        double p = uniform;
        if (a >= 0 && b <= 51 && a < b && last[combo_id(a, b)] >= 0) p = prob[combo_id(a, b)];
        const double old = w[i];
        double nw = old * p;
        if (nw < kWeightFloor && old > 0.0) nw = kWeightFloor;
        w[i] = nw;
        mx = nw > mx ? nw : mx;
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    mx = -1.0;
    for (int i = 0; i < kNarrowThreads / 32; ++i) mx = fmax(mx, red[i]);
    if (mx > 0.0)
        for (int i = tid; i < n; i += blockDim.x) w[i] = w[i] / mx;
    if (tid == 0) *applied = 1;
}

#define NCK(call)                                                                     \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            set_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #call); \
            rc = e_ == cudaErrorMemoryAllocation ? SS_ERR_NOMEM : SS_ERR_CUDA;        \
            goto done;                                                                \
        }                                                                             \
    } while (0)

}  // namespace

int session_narrow(Session *s, int player, int node, unsigned action_mask, int n, const int *hand_cards,
                   double *weights, int *applied) {
    const Plan &P = s->P;
    if (player < 0 || player >= P.np || n < 0 || (n > 0 && (!hand_cards || !weights))) {
        set_error("ss_session_narrow: bad player or range arrays");
        return SS_ERR_INVALID;
    }
    int di = -1;
    for (int i = 0; i < P.num_dec; ++i) {
        const int x = P.dec_nodes[i];
        if (node >= 0 ? x == node : s->dec_player_host[i] == player) {
            di = i;
            break;
        }
    }
    if (di < 0 || s->dec_player_host[di] != player) {
        set_error("ss_session_narrow: node is not a decision node of the player");
        return SS_ERR_INVALID;
    }
    const int x = P.dec_nodes[di];
    const int fe = P.first_edge[x], na = s->dec_na_host[di];
    if (action_mask == 0 || (na < 32 && (action_mask >> na) != 0)) {
        set_error("ss_session_narrow: action mask outside the node's actions");
        return SS_ERR_INVALID;
    }
    int rc = SS_OK;
    char *buf = nullptr;
    int flag = 0;
    const size_t cb = static_cast<size_t>(n) * 2 * sizeof(int), wb = static_cast<size_t>(n) * sizeof(double);
    const size_t wo = (cb + 15) / 16 * 16, fo = wo + (wb + 15) / 16 * 16;
    if (cudaSetDevice(s->device) != cudaSuccess) {
        set_error("ss_session_narrow: cudaSetDevice failed");
        return SS_ERR_CUDA;
    }
    NCK(cudaMallocAsync(reinterpret_cast<void **>(&buf), fo + 16, s->stream));
    if (n > 0) {
        NCK(cudaMemcpyAsync(buf, hand_cards, cb, cudaMemcpyHostToDevice, s->stream));
        NCK(cudaMemcpyAsync(buf + wo, weights, wb, cudaMemcpyHostToDevice, s->stream));
    }
    k_narrow<<<1, kNarrowThreads, 0, s->stream>>>(s->c, player, fe, na, action_mask,
                                                 reinterpret_cast<const int *>(buf),
                                                 reinterpret_cast<double *>(buf + wo), n,
                                                 reinterpret_cast<int *>(buf + fo));
    NCK(cudaGetLastError());
    if (n > 0) NCK(cudaMemcpyAsync(weights, buf + wo, wb, cudaMemcpyDeviceToHost, s->stream));
    NCK(cudaMemcpyAsync(&flag, buf + fo, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    NCK(cudaStreamSynchronize(s->stream));
    if (applied) *applied = flag;
done:
    if (buf) {
        cudaFreeAsync(buf, s->stream);
        cudaStreamSynchronize(s->stream);
    }
    return rc;
}

}  // namespace ssb
