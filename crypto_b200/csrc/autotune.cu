// Autotuner: per size class (log2 n) and curve, time on this GPU the
// candidate MSM window widths around the cost model's choice (256-bit
// windows and the windows of GLV halves), the candidate NTT radix splits,
// and -- with a resident SRS -- the shifted-table window of single KZG
// commits (13, 16 or 19 bits, which the batched and served commits use per
// commit); keep the fastest and cache them in a text file keyed by GPU name
// and driver version.  Plans consult the tables first (msm_tune_get,
// ntt_tune_get, commit_tune_get), falling back to the cost models.
#include "../../include/kinet_b200/crypto_b200.h"
#include "kzg.cuh"
#include "msm.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>
#include <string>
#include <vector>

namespace kb200 {

static std::string device_key() {
    int dev = 0, drv = 0;
    KB_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    KB_CUDA(cudaGetDeviceProperties(&prop, dev));
    KB_CUDA(cudaDriverGetVersion(&drv));
    std::string name = prop.name;
    for (char& ch : name)
        if (ch == ' ') ch = '_';
    return name + "|" + std::to_string(drv);
}

// The choice among candidates: the default (the cost model's) unless the
// fastest candidate beats it by more than TUNE_MARGIN, so that timing noise
// on short runs does not move the choice from run to run.
constexpr float TUNE_MARGIN = 0.03f;
static int pick_fastest(int def, const std::vector<int>& cands, const std::function<float(int)>& time_of,
                        float* best_ms) {
    const float t_def = time_of(def);
    int best = def;
    float best_t = t_def;
    for (int c : cands) {
        if (c == def) continue;
        const float t = time_of(c);
        if (t < best_t) {
            best_t = t;
            best = c;
        }
    }
    if (best_t < t_def * (1.0f - TUNE_MARGIN)) {
        *best_ms = best_t;
        return best;
    }
    *best_ms = t_def;
    return def;
}

static float time_ms(cudaStream_t st, const std::function<void()>& fn, int reps) {
    cudaEvent_t a, b;
    KB_CUDA(cudaEventCreate(&a));
    KB_CUDA(cudaEventCreate(&b));
    fn();  // warm-up (plan + scratch)
    KB_CUDA(cudaStreamSynchronize(st));
    KB_CUDA(cudaEventRecord(a, st));
    for (int i = 0; i < reps; ++i) fn();
    KB_CUDA(cudaEventRecord(b, st));
    KB_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    KB_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
}

}  // namespace kb200

using namespace kb200;

extern "C" {

// Tune MSM windows for log2 sizes in [log_lo, log_hi] and NTT splits in the
// same range; append the results to cache_path (if non-null).  Returns the
// number of size classes tuned, or a negative error.
int kb200_autotune(uint32_t curve, int log_lo, int log_hi, const char* cache_path) {
    if ((curve != 1 && curve != 2) || log_lo < 0 || log_hi > 26 || log_lo > log_hi)
        return KB200_CRYPTO_ERR_INPUT;
    try {
        cudaStream_t st;
        KB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        const size_t nmax = (size_t)1 << log_hi;
        const int pb = curve == 2 ? 96 : 64;
        std::vector<uint8_t> hs(nmax * 32);
        kb200_gen_scalars((int)curve, 0xA17u, nmax, 0, hs.data());
        DevBuf sc, pts, table, out, nt;
        sc.reserve(nmax * 32, st);
        pts.reserve(nmax * pb, st);
        table.reserve(nmax * (size_t)table_words((int)curve) * 4, st);
        out.reserve(256, st);
        KB_CUDA(cudaMemcpyAsync(sc.ptr, hs.data(), nmax * 32, cudaMemcpyHostToDevice, st));
        FixedBase* fb = fixed_base_create((int)curve, st);
        fixed_base_mul(fb, sc.as<uint8_t>(), nmax, table.as<uint32_t>(), pts.as<uint8_t>(), st);
        MsmEngine* eng = msm_engine_create((int)curve);
        NttEngine* ntt = ntt_engine_create((int)curve);
        nt.reserve(nmax * 32, st);
        std::ostringstream log;
        const std::string key = device_key();
        int tuned = 0;
        for (int lg = log_lo; lg <= log_hi; ++lg) {
            const size_t n = (size_t)1 << lg;
            MsmOptions base;
            const int c0 = make_msm_plan((int)curve, n, base).c;
            const int reps = lg >= 20 ? 2 : (lg >= 16 ? 5 : 20);
            std::vector<int> cs;
            for (int c = std::max(4, c0 - 2); c <= std::min(20, c0 + 2); ++c) cs.push_back(c);
            float best = 0;
            const int best_c = pick_fastest(c0, cs, [&](int c) {
                MsmOptions o;
                o.force_c = c;
                return time_ms(st, [&] {
                    msm_run_table(eng, sc.as<uint8_t>(), table.as<uint32_t>(), n,
                                  out.as<uint8_t>(), nullptr, st, o);
                }, reps);
            }, &best);
            msm_tune_set((int)curve, lg, best_c, false);
            log << key << " msm " << curve << " " << lg << " " << best_c << " " << best << "\n";
            // windows of the GLV halves (the wire path with the G1 promise:
            // BN254 always splits, BLS12-381 on the _subgroup entry points)
            {
                MsmOptions g;
                g.points_in_g1 = true;
                const int g0 = make_msm_plan_glv((int)curve, n, g).c;
                std::vector<int> gs;
                for (int c = std::max(4, g0 - 2); c <= std::min(20, g0 + 2); ++c) gs.push_back(c);
                float best_gt = 0;
                const int best_g = pick_fastest(g0, gs, [&](int c) {
                    MsmOptions o;
                    o.force_c = c;
                    o.points_in_g1 = true;
                    return time_ms(st, [&] {
                        msm_run_wire(eng, sc.as<uint8_t>(), pts.as<uint8_t>(), n, out.as<uint8_t>(),
                                     nullptr, st, o);
                    }, reps);
                }, &best_gt);
                msm_tune_set((int)curve, lg, best_g, true);
                log << key << " msm_glv " << curve << " " << lg << " " << best_g << " " << best_gt << "\n";
            }
            // NTT first-pass radix (two- and three-pass sizes)
            if (lg > 12) {
                KB_CUDA(cudaMemcpyAsync(nt.ptr, sc.ptr, n * 32, cudaMemcpyDeviceToDevice, st));
                std::vector<int> cands;
                for (int r1 = 3; r1 <= 10; ++r1) {
                    const int rest = lg - r1;
                    if (lg <= 20 ? (rest >= 3 && rest <= 10) : (rest >= 6 && rest <= 20)) cands.push_back(r1);
                }
                // 0 = the planner's own split; short transforms get enough
                // repetitions for about a millisecond of work each
                const int nreps = lg <= 16 ? 40 : (lg <= 20 ? 8 : 3);
                float best_t = 0;
                const int best_r = pick_fastest(0, cands, [&](int r1) {
                    ntt_tune_set((int)curve, lg, r1);
                    return time_ms(st, [&] { ntt_run(ntt, nt.as<uint32_t>(), n, 0, 0, 1, st); }, nreps);
                }, &best_t);
                ntt_tune_set((int)curve, lg, best_r);
                log << key << " ntt " << curve << " " << lg << " " << best_r << " " << best_t << "\n";
            }
            ++tuned;
        }
        KB_CUDA(cudaStreamSynchronize(st));
        msm_engine_destroy(eng);
        ntt_engine_destroy(ntt);
        fixed_base_destroy(fb);
        for (DevBuf* b : {&sc, &pts, &table, &out, &nt}) b->release();
        cudaStreamDestroy(st);
        // shifted-table windows of single commits (BLS12-381, resident SRS)
        std::string commit_log;
        if (curve == 2) tune_commit_windows(log_lo, log_hi, key, commit_log);
        if (cache_path) {
            std::ofstream f(cache_path, std::ios::app);
            f << log.str() << commit_log;
        }
        return tuned;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return KB200_CRYPTO_ERR_BACKEND;
    }
}

// Apply cached entries whose GPU key matches this device.  Returns the number
// applied (0 if the file is absent), or a negative error.
int kb200_autotune_load(const char* cache_path) {
    if (!cache_path) return KB200_CRYPTO_ERR_INPUT;
    try {
        std::ifstream f(cache_path);
        if (!f) return 0;
        const std::string key = device_key();
        std::string line;
        int applied = 0;
        while (std::getline(f, line)) {
            std::istringstream is(line);
            std::string k, kind;
            int curve = 0, lg = 0, v = 0;
            if (!(is >> k >> kind >> curve >> lg >> v)) continue;
            if (k != key) continue;
            if (kind == "msm") {
                msm_tune_set(curve, lg, v, false);
                ++applied;
            } else if (kind == "msm_glv") {
                msm_tune_set(curve, lg, v, true);
                ++applied;
            } else if (kind == "ntt") {
                ntt_tune_set(curve, lg, v);
                ++applied;
            } else if (kind == "commit" && curve == 2) {
                commit_tune_set(lg, v);
                ++applied;
            }
        }
        return applied;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return KB200_CRYPTO_ERR_BACKEND;
    }
}

// Direct access to the tuning tables (also used by tests).
int kb200_tune_get(int kind, uint32_t curve, int log_n) {
    switch (kind) {
        case 0: return msm_tune_get((int)curve, log_n, false);
        case 1: return ntt_tune_get((int)curve, log_n);
        case 2: return msm_tune_get((int)curve, log_n, true);
        case 3: return curve == 2 ? commit_tune_get(log_n) : 0;
        default: return 0;
    }
}
void kb200_tune_set(int kind, uint32_t curve, int log_n, int value) {
    switch (kind) {
        case 0: msm_tune_set((int)curve, log_n, value, false); break;
        case 1: ntt_tune_set((int)curve, log_n, value); break;
        case 2: msm_tune_set((int)curve, log_n, value, true); break;
        case 3: if (curve == 2) commit_tune_set(log_n, value); break;
        default: break;
    }
}

}  // extern "C"
