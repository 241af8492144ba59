// apsm_detector: device state and the train / detect call sequences.
#include "apsm_host.hpp"
#include "apsm_kernels.cuh"
#include "apsm_gram.cuh"
#include "apsm_lls.cuh"

#include <algorithm>
#include <cstdlib>
#include <string>

using namespace apsm;

namespace {

uint32_t pow2_at_least(uint32_t x)
{
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

int env_int(const char* name, int dflt)
{
    const char* v = std::getenv(name);
    return v ? std::atoi(v) : dflt;
}

} // namespace

#define APSM_CK(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);                            \
    } while (0)

apsm_status apsm_detector::cuda_fail(cudaError_t e, const char* what)
{
    cudaGetLastError(); // clear a non-sticky error
    last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? APSM_ERR_OUT_OF_MEMORY : APSM_ERR_CUDA;
}

apsm_detector::~apsm_detector()
{
    if (stream) cudaStreamSynchronize(stream);
    gram_workspace_free(gram);
    lls_workspace_free(lls);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (auto& e : stage_ev)
        if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
}

ModelParams apsm_detector::model_params() const
{
    ModelParams mp;
    mp.wL = cfg.wL;
    mp.wG = cfg.wG;
    mp.ew = -0.5f / variance_eff;
    mp.eB = cfg.eB;
    return mp;
}

apsm_status apsm_detector::init(const Config& c, uint32_t num_antennas, uint32_t num_users)
{
    cfg = c;
    N = num_antennas;
    D = 2 * N;
    Dp = row_pitch(D);
    U = num_users;
    is_lls = cfg.otype == "LLS";
    cap = 2 * cfg.dict_size;
    // ApsmNomaDetector constructor (apsm_noma_detector.cu:79-80)
    variance_eff = cfg.variance;
    if (variance_eff != 0) variance_eff *= float(N * N);

    APSM_CK(cudaGetDevice(&device));
    cudaDeviceProp prop;
    APSM_CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        last_error = "an sm_100 (Blackwell) device is required, found sm_" + std::to_string(prop.major) +
                     std::to_string(prop.minor);
        return APSM_ERR_NO_DEVICE;
    }
    APSM_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    APSM_CK(cudaEventCreate(&ev0));
    APSM_CK(cudaEventCreate(&ev1));
    for (auto& e : stage_ev) APSM_CK(cudaEventCreate(&e));
    APSM_CK(dict_X.ensure(size_t(cap) * Dp));
    APSM_CK(dict_nrm.ensure(cap));
    APSM_CK(dict_y.ensure(size_t(U) * cap));
    APSM_CK(dict_a.ensure(size_t(U) * cap));
    APSM_CK(w.ensure(size_t(U) * D));
    APSM_CK(train_err.ensure(1));
    APSM_CK(cudaMemset(train_err.p, 0, sizeof(int)));
    cluster = env_int("APSM_TRAIN_CLUSTER", 16);
    gram_one_product = env_int("APSM_GRAM_ONE_PRODUCT", 0) != 0;
    force_glob_a = env_int("APSM_TRAIN_GLOBAL_RING", 0) != 0;
    return reset();
}

apsm_status apsm_detector::reset()
{
    // resetState (apsm_noma_detector.cu:89-93): fresh, zeroed training state.
    // Stream-ordered: work already enqueued sees the old state, later work the new.
    used = 0;
    APSM_CK(cudaMemsetAsync(dict_a.p, 0, sizeof(float) * size_t(U) * cap, stream));
    APSM_CK(cudaMemsetAsync(w.p, 0, sizeof(float) * size_t(U) * D, stream));
    return APSM_OK;
}

apsm_status apsm_detector::train(const float2* d_rx, const float2* d_tx, uint32_t P, cudaStream_t s, float* ms,
                                 HistoryRequest* hist)
{
    if (hist) hist->n_steps = 0;
    if (is_lls || cfg.lls_init) {
        // LlsNomaDetector::train (lls_detector.cu:136-161) on the unshuffled pilots;
        // for llsInitialization (apsm_noma_detector.cu:98-99, 331-346) w = w_lls / wL
        APSM_CK(uX.ensure(size_t(2 * P) * Dp));
        APSM_CK(uy.ensure(size_t(U) * 2 * P));
        dim3 grid((P + kPackSamples - 1) / kPackSamples);
        pack_rows_kernel<<<grid, 256, sizeof(float2) * N * kPackSamples, s>>>(d_rx, int(N), int(P), nullptr, uX.p,
                                                                            int(Dp), 0, nullptr);
        APSM_CK(cudaGetLastError());
        gather_targets_kernel<<<(int(P * U) + 255) / 256, 256, 0, s>>>(d_tx, int(P), int(U), nullptr, uy.p,
                                                                      size_t(2 * P), 0);
        APSM_CK(cudaGetLastError());
        if (ms) APSM_CK(cudaEventRecord(ev0, s));
        apsm_status st = lls_solve(this, uX.p, int(2 * P), uy.p, size_t(2 * P), 0, is_lls ? 1.f : cfg.wL, s);
        if (st != APSM_OK) return st;
        if (is_lls) {
            used = 2 * P; // marks the detector as trained
            if (ms) {
                APSM_CK(cudaEventRecord(ev1, s));
                APSM_CK(cudaEventSynchronize(ev1));
                APSM_CK(cudaEventElapsedTime(ms, ev0, ev1));
            }
            return APSM_OK;
        }
        APSM_CK(cudaMemcpyAsync(w.p, lls_weights(this), sizeof(float) * size_t(U) * D, cudaMemcpyDeviceToDevice, s));
    }
    if (variance_eff == 0.f) {
        // computeGaussianVarianceHeuristic of the pilots (on the GPU; the multiset of pair
        // distances, hence the result, does not depend on the training shuffle)
        const size_t M = size_t(P) * (P - 1) / 2;
        APSM_CK(vh_nd.ensure(std::max<size_t>(M, 1)));
        APSM_CK(vh_hist.ensure(256));
        std::string err;
        apsm_status st = variance_heuristic_gpu(d_rx, N, P, vh_nd.p, vh_hist.p, s, &variance_eff, &err);
        if (st != APSM_OK) {
            last_error = err;
            return st;
        }
        if (!(variance_eff > 0.f)) {
            last_error = "Gaussian variance heuristic produced a non-positive variance";
            return APSM_ERR_INVALID_ARGUMENT;
        }
    }
    const ModelParams mp = model_params();
    const uint32_t rows_new = 2 * P;
    const uint32_t nU = used + rows_new;
    const uint32_t q2 = 2 * cfg.window;

    int final_hi = 0;
    std::vector<TrainStep> h_steps = build_schedule(cfg, used, P, cap, &final_hi);

    APSM_CK(uX.ensure(size_t(nU) * Dp));
    APSM_CK(unrm.ensure(nU));
    APSM_CK(uy.ensure(size_t(U) * nU));
    APSM_CK(ua.ensure(size_t(U) * nU));

    const int T_steps = int(h_steps.size());
    uint32_t hist_nE = 0;
    int hist_tiles = 0;
    if (hist && T_steps > 0) {
        if (uint32_t(T_steps) > hist->max_steps) {
            last_error = "train history: " + std::to_string(T_steps) + " steps, the output holds " +
                         std::to_string(hist->max_steps);
            return APSM_ERR_INVALID_ARGUMENT;
        }
        hist_nE = 2 * P + 2 * hist->S;
        hist_tiles = history_tiles(int(hist_nE));
        const size_t UT = size_t(U) * T_steps;
        const size_t floats = UT * (q2 + D + nU + size_t(hist_tiles) * 6) + size_t(U) * nU + size_t(hist_nE) * Dp +
                              size_t(U) * hist_nE;
        if (floats * sizeof(float) > (size_t(8) << 30)) {
            last_error = "train history needs " + std::to_string(floats * sizeof(float) >> 20) +
                         " MiB of scratch (steps x universe rows); more than the 8 GiB it may take";
            return APSM_ERR_UNSUPPORTED;
        }
        APSM_CK(h_snap_a.ensure(UT * q2));
        APSM_CK(h_snap_w.ensure(UT * D));
        APSM_CK(h_snap_scale.ensure(UT));
        APSM_CK(h_a0.ensure(size_t(U) * nU));
        APSM_CK(h_A.ensure(UT * nU));
        APSM_CK(h_E.ensure(size_t(hist_nE) * Dp));
        APSM_CK(h_Ey.ensure(size_t(U) * hist_nE));
        APSM_CK(h_part.ensure(UT * hist_tiles * 6));
    }

    const int* d_perm = nullptr;
    if (cfg.shuffle) {
        std::vector<int> pm = shuffle_permutation(P);
        APSM_CK(perm.ensure(P));
        APSM_CK(cudaMemcpyAsync(perm.p, pm.data(), sizeof(int) * P, cudaMemcpyHostToDevice, s));
        APSM_CK(cudaStreamSynchronize(s)); // pm is a local
        d_perm = perm.p;
    }

    // universe = dictionary rows already present, then the new pilots
    if (used > 0) {
        APSM_CK(cudaMemcpyAsync(uX.p, dict_X.p, sizeof(float) * size_t(used) * Dp, cudaMemcpyDeviceToDevice, s));
        APSM_CK(cudaMemcpyAsync(unrm.p, dict_nrm.p, sizeof(float) * used, cudaMemcpyDeviceToDevice, s));
        APSM_CK(cudaMemcpy2DAsync(uy.p, sizeof(float) * nU, dict_y.p, sizeof(float) * cap, sizeof(float) * used, U,
                                  cudaMemcpyDeviceToDevice, s));
        APSM_CK(cudaMemcpy2DAsync(ua.p, sizeof(float) * nU, dict_a.p, sizeof(float) * cap, sizeof(float) * used, U,
                                  cudaMemcpyDeviceToDevice, s));
    }
    APSM_CK(cudaMemset2DAsync(ua.p + used, sizeof(float) * nU, 0, sizeof(float) * rows_new, U, s));
    {
        dim3 grid((P + kPackSamples - 1) / kPackSamples);
        size_t sm = sizeof(float2) * N * kPackSamples;
        pack_rows_kernel<<<grid, 256, sm, s>>>(d_rx, int(N), int(P), d_perm, uX.p, int(Dp), int(used), unrm.p);
        APSM_CK(cudaGetLastError());
        int nt = int(P * U);
        gather_targets_kernel<<<(nt + 255) / 256, 256, 0, s>>>(d_tx, int(P), int(U), d_perm, uy.p, nU, int(used));
        APSM_CK(cudaGetLastError());
    }

    if (hist_nE > 0) // coefficients before the first step (rows of earlier calls; new rows 0)
        APSM_CK(cudaMemcpyAsync(h_a0.p, ua.p, sizeof(float) * size_t(U) * nU, cudaMemcpyDeviceToDevice, s));
    APSM_CK(cudaEventRecord(ev0, s));
    if (!h_steps.empty()) {
        const int T = int(h_steps.size());
        int v_first = h_steps[0].hi - h_steps[0].wk;
        for (const auto& st : h_steps) v_first = std::min(v_first, st.hi - st.wk);
        // normConstraint sums over every dictionary row's column, not only the window rows'
        if (cfg.norm_constraint > 0.f) v_first = 0;
        const int nV = int(nU) - v_first;
        // longest kernel column (rows column_base(v) .. min(nU, v + q2), 16-byte multiple)
        int Lk = 4;
        for (int v = v_first; v < int(nU); ++v) {
            int len = int(round_up(uint32_t(std::min<int>(int(nU), v + int(q2))), 4u)) - column_base(v, int(cap));
            Lk = std::max(Lk, len);
        }
        // rows in flight at once: window of step t-1 up to the rows fetched for t + kLookahead
        int span = 1, max_reveal = 0;
        for (int t = 0; t < T; ++t) {
            const int tp = std::max(0, t - 1), tn = std::min(T - 1, t + kLookahead);
            span = std::max(span, h_steps[tn].hi - (h_steps[tp].hi - h_steps[tp].wk));
            max_reveal = std::max(max_reveal, h_steps[t].hi - h_steps[t].reveal_lo);
        }
        APSM_CK(K.ensure(size_t(nV) * Lk));
        APSM_CK(steps.ensure(h_steps.size()));
        APSM_CK(cudaMemcpyAsync(steps.p, h_steps.data(), sizeof(TrainStep) * h_steps.size(), cudaMemcpyHostToDevice, s));
        {
            dim3 grid((Lk + kGramRows - 1) / kGramRows, (nV + kGramColsPerBlock - 1) / kGramColsPerBlock);
            gram_columns_kernel<<<grid, kGramRows, 0, s>>>(uX.p, int(Dp), int(D), int(nU), v_first, nV, Lk, int(cap),
                                                           mp, K.p);
            APSM_CK(cudaGetLastError());
        }
        TrainArgs ta;
        ta.X = uX.p;
        ta.nrm = unrm.p;
        ta.y = uy.p;
        ta.a = ua.p;
        ta.w = w.p;
        ta.K = K.p;
        ta.steps = steps.p;
        ta.n_steps = T;
        ta.nU = int(nU);
        ta.D = int(D);
        ta.Dp = int(Dp);
        ta.cap = int(cap);
        ta.q2 = int(q2);
        ta.Lk = Lk;
        ta.Lc = Lk;
        ta.v_first = v_first;
        ta.A_ring = int(pow2_at_least(cap + uint32_t(max_reveal) + 1));
        ta.XW = int(pow2_at_least(uint32_t(span) + 1));
        ta.used_before = int(used);
        ta.final_hi = final_hi;
        ta.y_stride = nU;
        ta.a_stride = nU;
        ta.mp = mp;
        ta.snap_a = hist_nE > 0 ? h_snap_a.p : nullptr;
        ta.snap_w = hist_nE > 0 ? h_snap_w.p : nullptr;
        ta.norm_c = cfg.norm_constraint;
        ta.a_glob = nullptr;
        ta.snap_scale = hist_nE > 0 && cfg.norm_constraint > 0.f ? h_snap_scale.p : nullptr;

        ta.XP = int(Dp) + 4; // padded window-row pitch (conflict-free column reads)
        ta.err = train_err.p;
        ta.users = int(U);
        ta.prof = prof_buffer;
        ta.NS = 0;

        // normConstraint rescales every coefficient after each step, which the incremental sweep's
        // running sums do not follow: such detectors train with the exact sweep
        if (cfg.train_incremental && !(cfg.norm_constraint > 0.f)) {
            // rows resident at once: window(t) and the rows entering at t+1 (and t+2 prefetched)
            int xs = 1;
            for (int t = 0; t < T; ++t) {
                const int t2 = std::min(T - 1, t + 1);
                xs = std::max(xs, h_steps[t2].hi - (h_steps[t].hi - h_steps[t].wk) + 1);
            }
            ta.XS = xs;
            // cluster size: the largest <= 8 of which every user gets one at once
            const int cmax = cluster > 0 ? std::min(16, cluster) : 8;
            {
                int bestC = 0;
                size_t bestSmem = 0;
                for (int C = cmax; C >= 1; C /= 2) {
                    const int nso = (xs + C - 1) / C + 1;
                    const int nsop = int(round_up(uint32_t(nso), 32u));
                    const size_t smem = incremental_smem_bytes(ta.XS, ta.XP, nsop, ta.A_ring);
                    if (smem > 227 * 1024) continue;
                    int mc = 0;
                    cudaError_t e = query_incremental_clusters(C, smem, int(U), &mc);
                    if (e != cudaSuccess) {
                        cudaGetLastError();
                        continue;
                    }
                    if (mc < 1) continue;
                    if (bestC == 0) {
                        bestC = C;
                        bestSmem = smem;
                    }
                    if (mc >= int(U)) {
                        bestC = C;
                        bestSmem = smem;
                        break;
                    }
                }
                if (bestC > 0) {
                    ta.NSO = (xs + bestC - 1) / bestC + 1;
                    ta.NSOp = int(round_up(uint32_t(ta.NSO), 32u));
                    int mc = 0;
                    APSM_CK(cudaMemsetAsync(train_err.p, 0, sizeof(int), s));
                    APSM_CK(cudaEventRecord(stage_ev[0], s));
                    APSM_CK(launch_train_incremental(bestC, bestSmem, s, ta, &mc));
                    APSM_CK(cudaEventRecord(stage_ev[1], s));
                    stage_valid[0] = true;
                    last_train_cluster = bestC;
                    last_train_staged = false;
                    last_train_glob_a = false;
                    goto sweep_done;
                }
            }
            // window too large for the incremental sweep's shared memory: the exact sweep below
        }

        // launch shape: the largest cluster (<= 16 CTAs) that holds its kernel
        // columns in shared memory and of which every user gets one at once
        // glob_a: the coefficient ring lives in global memory (one private copy per CTA)
        auto shape = [&](int C, bool staged, bool glob_a, int* nwarps_out, int* ns_out) -> size_t {
            int nwarps = std::max({(int(q2) + C - 1) / C, (int(D) * kWGroups + 31) / 32, 4});
            int ns = staged ? ta.XW / C + 2 : 0;
            *nwarps_out = nwarps;
            *ns_out = ns;
            return sizeof(float) * (size_t(ta.XW) * ta.XP + size_t(ns) * Lk + (glob_a ? 0 : size_t(ta.A_ring)) +
                                    kMaxFeatures + 2 * q2 + size_t(nwarps) * 32 + 2 * size_t(ta.XW) + 64) +
                   48;
        };
        const size_t smem_limit = 227 * 1024;
        struct Choice {
            int C = 0, nwarps = 0, ns = 0, clusters = 0;
            bool staged = false, glob_a = false;
            size_t smem = 0;
        } best;
        const int cmax = cluster > 0 ? std::min(16, cluster) : 16;
        // shared-memory coefficient ring first; a global one only when no shape holds it
        for (int ga = force_glob_a ? 1 : 0; ga < 2 && best.C == 0; ++ga) {
            for (int C = cmax; C >= 1; C /= 2) {
                for (int st = 1; st >= 0; --st) {
                    int nw = 0, ns = 0;
                    size_t sm = shape(C, st == 1, ga == 1, &nw, &ns);
                    if (sm > smem_limit || nw > 32) continue;
                    int mc = 0;
                    if (query_train_clusters(st == 1, ga == 1, C, nw * 32, sm, int(U), &mc) != cudaSuccess) {
                        cudaGetLastError();
                        continue;
                    }
                    if (mc < 1) continue;
                    // prefer: all users concurrent, then staged columns, then larger clusters
                    auto score = [&](int clusters, bool staged, int c) {
                        return (clusters >= int(U) ? 4 : 0) + (staged ? 2 : 0) + (c >= 8 ? 1 : 0);
                    };
                    if (best.C == 0 || score(mc, st == 1, C) > score(best.clusters, best.staged, best.C)) {
                        best.C = C;
                        best.nwarps = nw;
                        best.ns = ns;
                        best.clusters = mc;
                        best.staged = st == 1;
                        best.glob_a = ga == 1;
                        best.smem = sm;
                    }
                    break; // staged preferred at this cluster size
                }
                if (best.C != 0 && best.clusters >= int(U) && best.staged) break;
            }
        }
        if (best.C == 0) {
            last_error = "training kernel does not fit one cluster (window " + std::to_string(q2) +
                         " rows, dictionary " + std::to_string(cap) + " rows)";
            return APSM_ERR_UNSUPPORTED;
        }
        ta.NS = best.ns;
        ta.users = int(U);
        ta.prof = prof_buffer;
        if (best.glob_a) {
            APSM_CK(a_rings.ensure(size_t(U) * best.C * ta.A_ring));
            ta.a_glob = a_rings.p;
        }
        int max_clusters = 0;
        APSM_CK(cudaMemsetAsync(train_err.p, 0, sizeof(int), s));
        APSM_CK(cudaEventRecord(stage_ev[0], s));
        APSM_CK(launch_train_exact(best.staged, best.C, best.nwarps * 32, best.smem, s, ta, &max_clusters));
        APSM_CK(cudaEventRecord(stage_ev[1], s));
        stage_valid[0] = true;
        if (max_clusters < 1) {
            last_error = "training cluster of " + std::to_string(best.C) + " CTAs cannot be scheduled";
            return APSM_ERR_UNSUPPORTED;
        }
        last_train_cluster = best.C;
        last_train_staged = best.staged;
        last_train_glob_a = best.glob_a;
    }
sweep_done:
    if (hist_nE > 0) {
        // evaluation rows: this call's training rows (universe order), then the validation samples
        APSM_CK(cudaMemcpyAsync(h_E.p, uX.p + size_t(used) * Dp, sizeof(float) * size_t(rows_new) * Dp,
                                cudaMemcpyDeviceToDevice, s));
        APSM_CK(cudaMemcpy2DAsync(h_Ey.p, sizeof(float) * hist_nE, uy.p + used, sizeof(float) * nU,
                                  sizeof(float) * rows_new, U, cudaMemcpyDeviceToDevice, s));
        dim3 grid((hist->S + kPackSamples - 1) / kPackSamples);
        pack_rows_kernel<<<grid, 256, sizeof(float2) * N * kPackSamples, s>>>(hist->rx_val, int(N), int(hist->S),
                                                                            nullptr, h_E.p, int(Dp), int(rows_new),
                                                                            nullptr);
        APSM_CK(cudaGetLastError());
        const int nt = int(hist->S * U);
        gather_targets_kernel<<<(nt + 255) / 256, 256, 0, s>>>(hist->tx_val, int(hist->S), int(U), nullptr, h_Ey.p,
                                                               hist_nE, int(rows_new));
        APSM_CK(cudaGetLastError());
        HistoryArgs ha;
        ha.steps = steps.p;
        ha.n_steps = T_steps;
        ha.snap_a = h_snap_a.p;
        ha.snap_w = h_snap_w.p;
        ha.snap_scale = cfg.norm_constraint > 0.f ? h_snap_scale.p : nullptr;
        ha.a0 = h_a0.p;
        ha.a0_stride = nU;
        ha.used_before = int(used);
        ha.nU = int(nU);
        ha.cap = int(cap);
        ha.q2 = int(q2);
        ha.D = int(D);
        ha.Dp = int(Dp);
        ha.users = int(U);
        ha.A = h_A.p;
        ha.X = uX.p;
        ha.E = h_E.p;
        ha.Ey = h_Ey.p;
        ha.nE = int(hist_nE);
        ha.n_train = int(rows_new);
        ha.mp = mp;
        ha.bps = int(hist->bps);
        ha.mod_scale = hist->mod_scale;
        ha.rev_scale = float(1.0 / double(hist->mod_scale));
        ha.max_val = float((1u << (hist->bps / 2)) - 1u) * hist->mod_scale;
        ha.n_tiles = hist_tiles;
        ha.part = h_part.p;
        ha.out = hist->out;
        APSM_CK(launch_history(ha, s));
        hist->n_steps = uint32_t(T_steps);
    }
    APSM_CK(cudaEventRecord(ev1, s));

    // the dictionary after the sweep is the last min(final_hi, cap) universe rows
    const uint32_t used_new = std::min<uint32_t>(uint32_t(final_hi), cap);
    const uint32_t lo = uint32_t(final_hi) - used_new;
    if (used_new > 0) {
        APSM_CK(cudaMemcpyAsync(dict_X.p, uX.p + size_t(lo) * Dp, sizeof(float) * size_t(used_new) * Dp,
                                cudaMemcpyDeviceToDevice, s));
        APSM_CK(cudaMemcpyAsync(dict_nrm.p, unrm.p + lo, sizeof(float) * used_new, cudaMemcpyDeviceToDevice, s));
        APSM_CK(cudaMemcpy2DAsync(dict_y.p, sizeof(float) * cap, uy.p + lo, sizeof(float) * nU, sizeof(float) * used_new,
                                  U, cudaMemcpyDeviceToDevice, s));
        APSM_CK(cudaMemcpy2DAsync(dict_a.p, sizeof(float) * cap, ua.p + lo, sizeof(float) * nU, sizeof(float) * used_new,
                                  U, cudaMemcpyDeviceToDevice, s));
    }
    used = used_new;
    if (ms) {
        APSM_CK(cudaEventSynchronize(ev1));
        APSM_CK(cudaEventElapsedTime(ms, ev0, ev1));
    }
    return APSM_OK;
}

apsm_status apsm_detector::detect(const float2* d_rx, uint32_t S, float2* d_est, cudaStream_t s)
{
    const uint32_t ns = 2 * S;
    APSM_CK(xs.ensure(size_t(ns) * Dp));
    {
        dim3 grid((S + kPackSamples - 1) / kPackSamples);
        size_t sm = sizeof(float2) * N * kPackSamples;
        pack_rows_kernel<<<grid, 256, sm, s>>>(d_rx, int(N), int(S), nullptr, xs.p, int(Dp), 0, nullptr);
        APSM_CK(cudaGetLastError());
    }
    APSM_CK(cudaEventRecord(stage_ev[2], s));
    stage_valid[1] = true;
    if (is_lls) {
        apsm_status st = lls_detect(this, int(ns), reinterpret_cast<float*>(d_est), s);
        if (st != APSM_OK) return st;
        APSM_CK(cudaEventRecord(stage_ev[3], s));
        return APSM_OK;
    }
    if (cfg.detect_mode == DetectMode::Exact) {
        DetectArgs da;
        da.Xs = xs.p;
        da.n_samples = int(ns);
        da.Dp = int(Dp);
        da.D = int(D);
        da.dict = dict_X.p;
        da.M = int(used);
        da.a = dict_a.p;
        da.a_stride = cap;
        da.w = w.p;
        da.users = int(U);
        da.mp = model_params();
        da.out = reinterpret_cast<float*>(d_est);
        da.out_stride = ns;
        launch_detect_exact(da, s);
        APSM_CK(cudaGetLastError());
        APSM_CK(cudaEventRecord(stage_ev[3], s));
        return APSM_OK;
    }
    apsm_status st = detect_gram(this, S, reinterpret_cast<float*>(d_est), s);
    if (st != APSM_OK) return st;
    APSM_CK(cudaEventRecord(stage_ev[3], s));
    return APSM_OK;
}

apsm_status apsm_detector::train_host(const float2* rx, const float2* tx, uint32_t P, float* ms)
{
    APSM_CK(rx_stage.ensure(size_t(N) * P));
    APSM_CK(tx_stage.ensure(size_t(U) * P));
    APSM_CK(cudaMemcpyAsync(rx_stage.p, rx, sizeof(float2) * size_t(N) * P, cudaMemcpyHostToDevice, stream));
    APSM_CK(cudaMemcpyAsync(tx_stage.p, tx, sizeof(float2) * size_t(U) * P, cudaMemcpyHostToDevice, stream));
    float t = 0.f;
    apsm_status st = train(rx_stage.p, tx_stage.p, P, stream, &t);
    if (st != APSM_OK) return st;
    APSM_CK(cudaStreamSynchronize(stream));
    st = check_train_error();
    if (st != APSM_OK) return st;
    if (ms) *ms = t;
    return APSM_OK;
}

apsm_status apsm_detector::norm_ratio(uint32_t user, float* ratio)
{
    if (is_lls) {
        last_error = "the norm ratio belongs to APSM detectors";
        return APSM_ERR_UNSUPPORTED;
    }
    if (user >= U) {
        last_error = "user " + std::to_string(user) + " of a detector with " + std::to_string(U) + " users";
        return APSM_ERR_INVALID_ARGUMENT;
    }
    APSM_CK(nr_scratch.ensure(size_t(used) + 1));
    const ModelParams mp = model_params();
    APSM_CK(launch_norm_ratio(dict_X.p, int(Dp), int(D), int(used), dict_a.p + size_t(user) * cap, w.p + size_t(user) * D,
                              mp.ew, mp.wL, mp.wG, nr_scratch.p + 1, nr_scratch.p, stream));
    APSM_CK(cudaMemcpyAsync(ratio, nr_scratch.p, sizeof(float), cudaMemcpyDeviceToHost, stream));
    APSM_CK(cudaStreamSynchronize(stream));
    return APSM_OK;
}

uint32_t apsm_detector::train_steps(uint32_t P) const
{
    if (is_lls || P == 0) return 0;
    int final_hi = 0;
    return uint32_t(build_schedule(cfg, used, P, cap, &final_hi).size());
}

apsm_status apsm_detector::train_history_host(const float2* rx, const float2* tx, uint32_t P, const float2* rx_val,
                                              const float2* tx_val, uint32_t S, uint32_t bps, float mod_scale,
                                              float* history, uint32_t max_steps, uint32_t* n_steps, float* ms)
{
    const uint32_t T = train_steps(P);
    if (n_steps) *n_steps = T;
    if (T > max_steps) {
        last_error = "train history: " + std::to_string(T) + " steps, the output holds " + std::to_string(max_steps);
        return APSM_ERR_INVALID_ARGUMENT;
    }
    APSM_CK(rx_stage.ensure(size_t(N) * P));
    APSM_CK(tx_stage.ensure(size_t(U) * P));
    APSM_CK(h_rx.ensure(size_t(N) * S));
    APSM_CK(h_tx.ensure(size_t(U) * S));
    APSM_CK(h_out.ensure(size_t(U) * std::max<uint32_t>(T, 1) * 6));
    APSM_CK(cudaMemcpyAsync(rx_stage.p, rx, sizeof(float2) * size_t(N) * P, cudaMemcpyHostToDevice, stream));
    APSM_CK(cudaMemcpyAsync(tx_stage.p, tx, sizeof(float2) * size_t(U) * P, cudaMemcpyHostToDevice, stream));
    APSM_CK(cudaMemcpyAsync(h_rx.p, rx_val, sizeof(float2) * size_t(N) * S, cudaMemcpyHostToDevice, stream));
    APSM_CK(cudaMemcpyAsync(h_tx.p, tx_val, sizeof(float2) * size_t(U) * S, cudaMemcpyHostToDevice, stream));
    HistoryRequest req;
    req.rx_val = h_rx.p;
    req.tx_val = h_tx.p;
    req.S = S;
    req.bps = bps;
    req.mod_scale = mod_scale;
    req.out = h_out.p;
    req.max_steps = T;
    float t = 0.f;
    apsm_status st = train(rx_stage.p, tx_stage.p, P, stream, &t, &req);
    if (st != APSM_OK) return st;
    if (req.n_steps > 0)
        APSM_CK(cudaMemcpyAsync(history, h_out.p, sizeof(float) * size_t(U) * req.n_steps * 6, cudaMemcpyDeviceToHost,
                                stream));
    APSM_CK(cudaStreamSynchronize(stream));
    st = check_train_error();
    if (st != APSM_OK) return st;
    if (n_steps) *n_steps = req.n_steps;
    if (ms) *ms = t;
    return APSM_OK;
}

apsm_status apsm_detector::detect_host(const float2* rx, uint32_t S, float2* est, float* ms)
{
    APSM_CK(rx_stage.ensure(size_t(N) * S));
    APSM_CK(est_stage.ensure(size_t(U) * S));
    APSM_CK(cudaMemcpyAsync(rx_stage.p, rx, sizeof(float2) * size_t(N) * S, cudaMemcpyHostToDevice, stream));
    APSM_CK(cudaEventRecord(ev0, stream));
    apsm_status st = detect(rx_stage.p, S, est_stage.p, stream);
    if (st != APSM_OK) return st;
    APSM_CK(cudaEventRecord(ev1, stream));
    APSM_CK(cudaMemcpyAsync(est, est_stage.p, sizeof(float2) * size_t(U) * S, cudaMemcpyDeviceToHost, stream));
    APSM_CK(cudaStreamSynchronize(stream));
    st = detect_gram_check(this);
    if (st != APSM_OK) return st;
    if (ms) APSM_CK(cudaEventElapsedTime(ms, ev0, ev1));
    return APSM_OK;
}

apsm_status apsm_detector::get_state(float* dict, float* a_out, float* w_out)
{
    APSM_CK(cudaStreamSynchronize(stream));
    if (dict && used > 0)
        APSM_CK(cudaMemcpy2D(dict, sizeof(float) * D, dict_X.p, sizeof(float) * Dp, sizeof(float) * D, used,
                             cudaMemcpyDeviceToHost));
    if (a_out && used > 0)
        APSM_CK(cudaMemcpy2D(a_out, sizeof(float) * used, dict_a.p, sizeof(float) * cap, sizeof(float) * used, U,
                             cudaMemcpyDeviceToHost));
    if (w_out) APSM_CK(cudaMemcpy(w_out, w.p, sizeof(float) * size_t(U) * D, cudaMemcpyDeviceToHost));
    return APSM_OK;
}

apsm_status apsm_detector::copy_state_from(const apsm_detector& src)
{
    if (is_lls || src.is_lls) {
        last_error = "state copies need two APSM detectors";
        return APSM_ERR_UNSUPPORTED;
    }
    if (src.device != device || src.N != N || src.U != U || src.cap != cap) {
        last_error = "state copy between detectors of different device, antennas, users or dictionarySize";
        return APSM_ERR_INVALID_ARGUMENT;
    }
    if (src.cfg.wL != cfg.wL || src.cfg.wG != cfg.wG) {
        last_error = "state copy between detectors of different kernel weights";
        return APSM_ERR_INVALID_ARGUMENT;
    }
    if (cfg.variance != 0.f && src.variance_eff != variance_eff) {
        last_error = "state copy between detectors of different gaussianKernelVariance";
        return APSM_ERR_INVALID_ARGUMENT;
    }
    APSM_CK(cudaStreamSynchronize(src.stream));
    const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
    APSM_CK(cudaMemcpyAsync(dict_X.p, src.dict_X.p, sizeof(float) * size_t(cap) * Dp, k, stream));
    APSM_CK(cudaMemcpyAsync(dict_nrm.p, src.dict_nrm.p, sizeof(float) * cap, k, stream));
    APSM_CK(cudaMemcpyAsync(dict_y.p, src.dict_y.p, sizeof(float) * size_t(U) * cap, k, stream));
    APSM_CK(cudaMemcpyAsync(dict_a.p, src.dict_a.p, sizeof(float) * size_t(U) * cap, k, stream));
    APSM_CK(cudaMemcpyAsync(w.p, src.w.p, sizeof(float) * size_t(U) * D, k, stream));
    used = src.used;
    if (src.variance_eff != 0.f) variance_eff = src.variance_eff;
    return APSM_OK;
}

apsm_status apsm_detector::stage_ms(float* sweep_ms, float* detect_ms)
{
    float* out[2] = {sweep_ms, detect_ms};
    for (int k = 0; k < 2; ++k) {
        if (!out[k]) continue;
        *out[k] = -1.f;
        if (!stage_valid[k]) continue;
        APSM_CK(cudaEventSynchronize(stage_ev[2 * k + 1]));
        APSM_CK(cudaEventElapsedTime(out[k], stage_ev[2 * k], stage_ev[2 * k + 1]));
    }
    return APSM_OK;
}

apsm_status apsm_detector::check_train_error()
{
    int e = 0;
    APSM_CK(cudaMemcpy(&e, train_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        last_error = "training sweep gave up waiting for its cluster (bounded wait expired)";
        return APSM_ERR_CUDA;
    }
    return APSM_OK;
}
