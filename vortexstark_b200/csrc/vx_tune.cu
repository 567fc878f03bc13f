// Autotuner: picks, per device, the NTT pass plan of every transform length
// and the Merkle leaf-kernel subtree size of every tree depth by timing the
// candidates on scratch buffers of that size.  The knobs only change how the
// work is split into launches and threads; every choice computes the same
// values (the tests prove each plan against the oracle), so proofs stay
// byte-identical whatever the tuner picks.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vx_common.cuh"
#include "vx_fri.cuh"
#include "vx_merkle.cuh"
#include "vx_ntt.cuh"

using namespace vx;

namespace {

struct Scratch {
    void *p = nullptr;
    ~Scratch() { if (p) cudaFree(p); }
};

// Median of `reps` timed runs of fn on `st` after two untimed ones.
template <class F>
float time_ms(F fn, cudaStream_t st, int reps, cudaError_t *err) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    std::vector<float> t;
    for (int r = 0; r < reps + 2 && *err == cudaSuccess; r++) {
        cudaEventRecord(a, st);
        *err = fn();
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (r >= 2) t.push_back(ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (t.empty()) return 1e30f;
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

}  // namespace

extern "C" int vx_tune_set(uint32_t kind, uint32_t layers, uint32_t a, uint32_t b) {
    int dev = 0;
    VX_CUDA_TRY(cudaGetDevice(&dev));
    VX_CHECK_ARG(layers < 32, "vx_tune_set: layers %u >= 32", layers);
    if (kind == 0) {
        // a = 0 restores the default; a bottom pass of at least 9 layers lets
        // every upper pass's columns fit between its rows
        VX_CHECK_ARG(a == 0 || (a >= 9 && a <= 14 && b >= 3 && b <= 12),
                     "vx_tune_set: NTT plan needs bottom 9..14 and upper 3..12 (or 0 for the default)");
        ntt_knobs_set(dev, layers, a, b);
    } else if (kind == 1 || kind == 2) {
        VX_CHECK_ARG(a <= 4, "vx_tune_set: leaf subtree log must be 0 (default) .. 4");
        tree_knob_set(dev, layers, a, kind == 1 ? kLeafNarrow : kLeafFold);
    } else {
        VX_CHECK_ARG(false, "vx_tune_set: kind %u is not 0 (NTT plan), 1 (leaf subtree) or 2 (fold-leaf subtree)",
                     kind);
    }
    return VX_OK;
}

extern "C" int vx_tune_get(uint32_t kind, uint32_t layers, uint32_t *a, uint32_t *b) {
    VX_CHECK_ARG(a != nullptr && b != nullptr && layers < 32, "vx_tune_get: bad arguments");
    if (kind == 0) {
        ntt_knobs_get(layers, a, b);
    } else if (kind == 1 || kind == 2) {
        *a = tree_leaf_k(layers, kind == 1 ? kLeafNarrow : kLeafFold);
        *b = 0;
    } else {
        VX_CHECK_ARG(false, "vx_tune_get: kind %u is not 0, 1 or 2", kind);
    }
    return VX_OK;
}

extern "C" int vx_ntt_plan(uint32_t total, uint32_t bottom_max, uint32_t upper_max, uint32_t starts[32],
                           uint32_t layers[32], uint32_t tile_cols_log[32], uint32_t *n_passes) {
    VX_CHECK_ARG(total >= 4 && total <= 31, "vx_ntt_plan: total %u outside 4..31", total);
    VX_CHECK_ARG(bottom_max >= 9 && bottom_max <= 14 && upper_max >= 3 && upper_max <= 12,
                 "vx_ntt_plan: bottom 9..14 and upper 3..12");
    VX_CHECK_ARG(starts && layers && tile_cols_log && n_passes, "vx_ntt_plan: null output");
    *n_passes = ntt_plan(total, bottom_max, upper_max, starts, layers, tile_cols_log);
    return VX_OK;
}

extern "C" int vx_autotune(uint32_t max_log, char *report, size_t cap) {
    VX_CHECK_ARG(max_log >= 12 && max_log <= 28, "vx_autotune: max_log %u outside 12..28", max_log);
    int dev = 0;
    VX_CUDA_TRY(cudaGetDevice(&dev));
    const uint64_t n = 1ull << max_log;
    // data (n words), line + circle tables (2n words), a Merkle pool (the
    // largest is the one with one leaf pair per thread)
    // every region starts on a 64-word (256-byte) boundary: the fold leaves
    // read their inputs as 8-byte pairs, and a pool size can be odd
    auto a64 = [](uint64_t w) { return (w + 63) & ~63ull; };
    const uint64_t pool_max = a64(tree_pool_words(max_log, 1));
    // fold-leaf trees up to depth 25 (the first FRI layer of a 2^26-point
    // proof): 4 input columns of 2^(d+1) words, twiddles, 4 output columns
    const uint32_t fold_max = max_log < 25 ? max_log : 25;
    const uint64_t nf = 1ull << fold_max;
    Scratch sc;
    const uint64_t words = 3 * n + pool_max + 8 * nf + 4 * nf + nf + 64;
    VX_CUDA_TRY(cudaMalloc(&sc.p, words * 4));
    uint32_t *data = (uint32_t *)sc.p, *tab = data + n, *pool = tab + 2 * n;
    uint32_t *fin = pool + pool_max, *fout = fin + 8 * nf, *ftw = fout + 4 * nf, *falpha = ftw + nf;
    VX_CUDA_TRY(cudaMemset(sc.p, 0, words * 4));
    cudaStream_t st = nullptr;
    cudaError_t err = cudaSuccess;
    std::string js = "{\"ntt\":{";
    // ---- NTT pass plans ----
    for (uint32_t total = 13; total <= max_log && err == cudaSuccess; total++) {  // <= 12: one pass
        NttTables tw{tab, tab + n, {}, 0u};
        ntt_table_offsets(total, tw.off);
        float best = 1e30f;
        uint32_t bb = 11, bu = 8;
        std::vector<std::vector<uint32_t>> seen;
        // 4096-element tiles only: the larger tiles (bottom passes of 13-14
        // layers, upper passes of 10-12) can win this timing of an L2-resident
        // transform and then lose inside proofs, where the LDE's data is in
        // HBM; they stay available through vx_tune_set
        for (uint32_t bottom = 10; bottom <= 12; bottom++)
            for (uint32_t upper = 6; upper <= 9; upper++) {
                uint32_t ps[32], pr[32], pw[32];
                uint32_t np = ntt_plan(total, bottom, upper, ps, pr, pw);
                std::vector<uint32_t> key(pr, pr + np);
                if (std::find(seen.begin(), seen.end(), key) != seen.end()) continue;  // same plan
                seen.push_back(key);
                float ms = time_ms(
                    [&] {
                        return ntt_transform_planned(data, nullptr, 0, 1, total, tw, true, nullptr, 0, bottom, upper, st);
                    },
                    st, 5, &err);
                if (ms < best) { best = ms; bb = bottom; bu = upper; }
            }
        ntt_knobs_set(dev, total, bb, bu);
        char buf[96];
        snprintf(buf, sizeof(buf), "%s\"%u\":[%u,%u,%.4f]", total == 13 ? "" : ",", total, bb, bu, best);
        js += buf;
    }
    js += "},\"leaf_k\":{";
    // ---- Merkle leaf-subtree sizes ----
    for (uint32_t depth = 17; depth <= max_log && err == cudaSuccess; depth++) {
        float best = 1e30f;
        uint32_t bk = 0;
        for (uint32_t k = 1; k <= 4; k++) {
            if (depth - k < 13) continue;  // keep at least 2^13 threads
            TreeLevels lv;
            tree_plan(depth, pool, &lv, k);
            if ((err = tree_reset(lv, st)) != cudaSuccess) break;
            float ms = time_ms([&] { return tree_build(LeafM31{data}, lv, ChanStep{nullptr, nullptr, nullptr}, st); },
                               st, 3, &err);
            if (ms < best) { best = ms; bk = k; }
        }
        tree_knob_set(dev, depth, bk);
        char buf[96];
        snprintf(buf, sizeof(buf), "%s\"%u\":[%u,%.4f]", depth == 17 ? "" : ",", depth, bk, best);
        js += buf;
    }
    js += "},\"fold_leaf_k\":{";
    // ---- leaf-subtree sizes of fold-leaf (FRI layer) trees ----
    for (uint32_t depth = 17; depth <= fold_max && err == cudaSuccess; depth++) {
        float best = 1e30f;
        uint32_t bk = 0;
        const uint64_t m = 1ull << depth;
        LeafFold lf{fin, fin + 2 * m, fin + 4 * m, fin + 6 * m, ftw, falpha,
                    fout, fout + m, fout + 2 * m, fout + 3 * m, {}};
        for (uint32_t k = 1; k <= 4; k++) {
            TreeLevels lv;
            tree_plan(depth, pool, &lv, k);
            if ((err = tree_reset(lv, st)) != cudaSuccess) break;
            float ms = time_ms([&] { return tree_build(lf, lv, ChanStep{nullptr, nullptr, nullptr}, st); }, st, 3, &err);
            if (ms < best) { best = ms; bk = k; }
        }
        tree_knob_set(dev, depth, bk, kLeafFold);
        char buf[96];
        snprintf(buf, sizeof(buf), "%s\"%u\":[%u,%.4f]", depth == 17 ? "" : ",", depth, bk, best);
        js += buf;
    }
    js += "}}";
    if (err != cudaSuccess) {
        for (uint32_t l = 0; l < 32; l++) {  // back to the defaults
            ntt_knobs_set(dev, l, 0, 0);
            tree_knob_set(dev, l, 0, kLeafNarrow);
            tree_knob_set(dev, l, 0, kLeafFold);
        }
        set_last_error(VX_ERR_CUDA, "vx_autotune: %s", cudaGetErrorString(err));
        return VX_ERR_CUDA;
    }
    if (report && cap) {
        strncpy(report, js.c_str(), cap - 1);
        report[cap - 1] = 0;
    }
    return VX_OK;
}
