// ref_driver.cu — TEST INFRASTRUCTURE ONLY (oracle side, never shipped).
//
// Drives the reference's own CUDA launchers, compiled from the reference's
// sources by oracle/build_ref.sh into oracle/_ref/libvxref.so, through the
// orchestration of src/prover.rs:264-619 (prove_lean_inner), and writes the
// proof in the stark_cli.rs:1092-1123 layout.  Host-side pieces that are Rust
// in the reference (the transcript, coset constants, serialisation) come from
// the C oracle (vx_oracle.c) linked into the same library.  The point is to
// pin the oracle and the product against the reference's device arithmetic:
// NTT and twiddle conventions, Blake2s trees, quotient and folds.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <array>
#include <vector>

#include "vx_oracle.h"

extern "C" {
// reference launchers (src/cuda/ffi.rs)
void cuda_circle_ntt_evaluate(uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *,
                              uint32_t, uint32_t);
void cuda_circle_ntt_interpolate(uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *,
                                 uint32_t, uint32_t);
void cuda_compute_coset_points(uint32_t, uint32_t, uint32_t, uint32_t, uint32_t *, uint32_t *, uint32_t);
void cuda_extract_and_squash(const uint32_t *, uint32_t *, uint32_t *, uint32_t);
void cuda_batch_inverse_m31(const uint32_t *, uint32_t *, uint32_t);
void cuda_compute_fold_twiddle_sources(uint32_t, uint32_t, uint32_t, uint32_t, uint32_t *, uint32_t, uint32_t, int);
void cuda_zero_pad(const uint32_t *, uint32_t *, uint32_t, uint32_t);
void cuda_fibonacci_quotient(const uint32_t *, uint32_t *, uint32_t *, uint32_t *, uint32_t *, const uint32_t *,
                             uint32_t);
void cuda_merkle_hash_leaves_forge_single(const uint32_t *, uint32_t *, uint32_t);
void cuda_merkle_hash_leaves_forge_quad(const uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *,
                                        uint32_t *, uint32_t);
void cuda_merkle_hash_nodes(const uint32_t *, uint32_t *, uint32_t);
void cuda_merkle_reduce_to_root(const uint32_t *, uint32_t *, uint32_t);
void cuda_merkle_commit_small_soa4(const uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *, uint32_t *,
                                   uint32_t);
void cuda_merkle_tiled_soa4(const uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *, uint32_t *,
                            uint32_t);
void cuda_merkle_tiled_generic(const uint32_t *const *, uint32_t *, uint32_t, uint32_t);
void cuda_fold_line_soa(const uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *,
                        uint32_t *, uint32_t *, uint32_t *, uint32_t *, const uint32_t *, uint32_t);
void cuda_fold_circle_into_line_soa(uint32_t *, uint32_t *, uint32_t *, uint32_t *, const uint32_t *,
                                    const uint32_t *, const uint32_t *, const uint32_t *, const uint32_t *,
                                    const uint32_t *, const uint32_t *, uint32_t);
}

namespace {

struct Dev {
    uint32_t *p = nullptr;
    size_t n = 0;
    explicit Dev(size_t words) : n(words) { cudaMalloc(&p, (words ? words : 1) * 4); }
    ~Dev() { cudaFree(p); }
    Dev(const Dev &) = delete;
    Dev &operator=(const Dev &) = delete;
    std::vector<uint32_t> host(size_t words = 0) const {
        std::vector<uint32_t> h(words ? words : n);
        cudaMemcpy(h.data(), p, h.size() * 4, cudaMemcpyDeviceToHost);
        return h;
    }
};

// circle.rs:454-550 — forward (inverse) twiddles through the reference launchers.
void twiddles(const vxo_coset &c, bool inverse, Dev &line, Dev &circle, std::vector<uint32_t> &offs,
              std::vector<uint32_t> &sizes) {
    uint32_t n = 1u << c.log_size, half = n / 2;
    Dev x(n), y(n);
    cuda_compute_coset_points(c.initial.x, c.initial.y, c.step.x, c.step.y, x.p, y.p, n);
    cudaDeviceSynchronize();
    Dev fl(n - 1), fc(half);
    cudaMemcpy(fc.p, y.p, half * 4, cudaMemcpyDeviceToDevice);
    std::vector<Dev *> keep;
    uint32_t *cur = x.p, cur_n = n, off = 0;
    for (uint32_t l = 0; l + 1 < c.log_size; l++) {
        uint32_t ls = cur_n / 2;
        offs.push_back(off);
        sizes.push_back(ls);
        Dev *sq = new Dev(ls);
        cuda_extract_and_squash(cur, fl.p + off, sq->p, ls);
        cudaDeviceSynchronize();
        keep.push_back(sq);
        off += ls;
        cur = sq->p;
        cur_n = ls;
    }
    if (inverse) {
        cuda_batch_inverse_m31(fl.p, line.p, n - 1);
        cuda_batch_inverse_m31(fc.p, circle.p, half);
    } else {
        cudaMemcpy(line.p, fl.p, (n - 1) * 4, cudaMemcpyDeviceToDevice);
        cudaMemcpy(circle.p, fc.p, half * 4, cudaMemcpyDeviceToDevice);
    }
    cudaDeviceSynchronize();
    for (auto *d : keep) delete d;
}

// fri.rs:112-139
void fold_twiddles(const vxo_coset &c, bool extract_y, Dev &out) {
    uint32_t n = 1u << c.log_size;
    Dev src(n / 2);
    cuda_compute_fold_twiddle_sources(c.initial.x, c.initial.y, c.step.x, c.step.y, src.p, n, c.log_size,
                                      extract_y ? 1 : 0);
    cuda_batch_inverse_m31(src.p, out.p, n / 2);
    cudaDeviceSynchronize();
}

// Full tree with every level (merkle.rs:28-130 with the default forge-blake2s
// leaf kernels); levels[0] = leaves.
std::vector<std::vector<uint32_t>> full_tree(const uint32_t *const cols[], int ncols, uint32_t log_n) {
    uint32_t n = 1u << log_n;
    std::vector<std::vector<uint32_t>> lv;
    Dev leaves((size_t)n * 8);
    if (ncols == 1) cuda_merkle_hash_leaves_forge_single(cols[0], leaves.p, n);
    else cuda_merkle_hash_leaves_forge_quad(cols[0], cols[1], cols[2], cols[3], leaves.p, n);
    cudaDeviceSynchronize();
    lv.push_back(leaves.host());
    Dev *cur = nullptr;
    const uint32_t *src = leaves.p;
    for (uint32_t sz = n / 2; sz >= 1; sz /= 2) {
        Dev *par = new Dev((size_t)sz * 8);
        cuda_merkle_hash_nodes(src, par->p, sz);
        cudaDeviceSynchronize();
        lv.push_back(par->host());
        delete cur;
        cur = par;
        src = par->p;
        if (sz == 1) break;
    }
    delete cur;
    return lv;
}

// Root-only commitments of prove_lean (merkle.rs:142-383); must agree with
// the full tree's root.
void root_only(const uint32_t *const cols[], int ncols, uint32_t log_n, uint32_t root[8]) {
    uint32_t n = 1u << log_n;
    Dev r(8);
    if (ncols == 4 && n <= 2048) {
        cuda_merkle_commit_small_soa4(cols[0], cols[1], cols[2], cols[3], r.p, n);
    } else if (n >= 1024) {
        uint32_t tiles = n / 1024;
        Dev sub((size_t)tiles * 8);
        if (ncols == 4) {
            cuda_merkle_tiled_soa4(cols[0], cols[1], cols[2], cols[3], sub.p, n);
        } else {
            Dev ptrs(2);
            cudaMemcpy(ptrs.p, cols, sizeof(uint32_t *), cudaMemcpyHostToDevice);
            cuda_merkle_tiled_generic((const uint32_t *const *)ptrs.p, sub.p, 1, n);
            cudaDeviceSynchronize();
        }
        std::vector<Dev *> keep;
        const uint32_t *cur = sub.p;
        uint32_t size = tiles;
        while (size > 1024) {
            Dev *par = new Dev((size_t)(size / 2) * 8);
            cuda_merkle_hash_nodes(cur, par->p, size / 2);
            keep.push_back(par);
            cur = par->p;
            size /= 2;
        }
        if (size > 1) cuda_merkle_reduce_to_root(cur, r.p, size);
        else cudaMemcpy(r.p, cur, 32, cudaMemcpyDeviceToDevice);
        cudaDeviceSynchronize();
        for (auto *d : keep) delete d;
    } else {
        auto lv = full_tree(cols, ncols, log_n);
        memcpy(root, lv.back().data(), 32);
        return;
    }
    cudaDeviceSynchronize();
    auto h = r.host();
    memcpy(root, h.data(), 32);
}

struct W {
    std::vector<uint32_t> w;
    void u(uint32_t v) { w.push_back(v); }
    void s(const uint32_t *p, size_t k) { w.insert(w.end(), p, p + k); }
};

void decom(W &out, const std::vector<std::vector<uint32_t>> &lv, const std::vector<const std::vector<uint32_t> *> &cols,
           const std::vector<uint64_t> &idx) {
    uint32_t depth = (uint32_t)lv.size() - 1;
    out.u((uint32_t)idx.size());
    for (uint64_t i : idx) for (auto *c : cols) out.u((*c)[i]);
    for (uint64_t i : idx) for (auto *c : cols) out.u((*c)[i ^ 1]);
    for (int sib = 0; sib < 2; sib++)
        for (uint64_t i0 : idx) {
            uint64_t i = i0 ^ (uint64_t)sib;
            out.u(depth);
            for (uint32_t l = 0; l < depth; l++) {
                out.s(&lv[l][8 * (i ^ 1)], 8);
                i >>= 1;
            }
        }
}

}  // namespace

extern "C" int vxref_prove(uint32_t a, uint32_t b, uint32_t log_n, uint32_t blowup, uint32_t nq, uint8_t *out,
                           size_t cap, size_t *out_len) {
    uint32_t le = log_n + blowup;
    if (log_n < 4 || le > 24) return 1;  // full trees are kept on the host: small sizes only
    uint32_t n = 1u << log_n, N = 1u << le;
    // trace (air.rs:28-45) and upload
    std::vector<uint32_t> tr(n);
    tr[0] = a; tr[1] = b;
    for (uint32_t i = 2; i < n; i++) { uint32_t s = tr[i - 1] + tr[i - 2]; tr[i] = s >= VXO_P ? s - VXO_P : s; }
    Dev dtr(n);
    cudaMemcpy(dtr.p, tr.data(), n * 4, cudaMemcpyHostToDevice);
    // interpolate on half_coset(log_n)
    {
        Dev il(n - 1), ic(n / 2);
        std::vector<uint32_t> offs, sizes;
        twiddles(vxo_coset_half_coset(log_n), true, il, ic, offs, sizes);
        cuda_circle_ntt_interpolate(dtr.p, il.p, ic.p, offs.data(), sizes.data(), log_n - 1, n);
    }
    // zero-pad + evaluate on the eval domain
    Dev ev(N);
    cuda_zero_pad(dtr.p, ev.p, n, N);
    vxo_coset edom = le <= 30 ? vxo_coset_half_coset(le) : vxo_coset_subgroup(le);
    {
        Dev fl(N - 1), fc(N / 2);
        std::vector<uint32_t> offs, sizes;
        twiddles(edom, false, fl, fc, offs, sizes);
        cuda_circle_ntt_evaluate(ev.p, fl.p, fc.p, offs.data(), sizes.data(), le - 1, N);
    }
    std::vector<uint32_t> evh = ev.host();
    const uint32_t *tcols[1] = {ev.p};
    auto ttree = full_tree(tcols, 1, le);
    uint32_t troot[8], chk[8];
    memcpy(troot, ttree.back().data(), 32);
    root_only(tcols, 1, le, chk);
    if (memcmp(troot, chk, 32)) return 2;
    vxo_channel ch;
    vxo_channel_init(&ch);
    vxo_channel_mix_digest(&ch, troot);
    uint32_t alpha[4];
    vxo_channel_draw_felt(&ch, alpha);
    // quotient (constraint.cu:94-106) and its commitment
    Dev q0(N), q1(N), q2(N), q3(N);
    cuda_fibonacci_quotient(ev.p, q0.p, q1.p, q2.p, q3.p, alpha, N);
    cudaDeviceSynchronize();
    const uint32_t *qcols[4] = {q0.p, q1.p, q2.p, q3.p};
    auto qtree = full_tree(qcols, 4, le);
    uint32_t qroot[8];
    memcpy(qroot, qtree.back().data(), 32);
    root_only(qcols, 4, le, chk);
    if (memcmp(qroot, chk, 32)) return 3;
    std::vector<uint32_t> qh[4] = {q0.host(), q1.host(), q2.host(), q3.host()};
    vxo_channel_mix_digest(&ch, qroot);
    // FRI: circle fold, then line folds down to 2^3 (prover.rs:375-553)
    uint32_t nfri = le - 3;
    std::vector<std::vector<std::vector<uint32_t>>> ftrees;
    std::vector<std::array<std::vector<uint32_t>, 4>> fvals;
    std::vector<uint32_t> froots;
    uint32_t fa[4], fa2[4];
    vxo_channel_draw_felt(&ch, fa);
    vxo_qm31_mul(fa, fa, fa2);
    Dev *cur[4];
    for (int c = 0; c < 4; c++) { cur[c] = new Dev(N / 2); cudaMemset(cur[c]->p, 0, (N / 2) * 4); }
    {
        Dev tw(N / 2);
        fold_twiddles(edom, true, tw);
        cuda_fold_circle_into_line_soa(cur[0]->p, cur[1]->p, cur[2]->p, cur[3]->p, q0.p, q1.p, q2.p, q3.p, tw.p, fa,
                                       fa2, N / 2);
        cudaDeviceSynchronize();
    }
    uint32_t cl = le - 1;
    for (uint32_t k = 0; k < nfri; k++) {
        if (k > 0) {
            uint32_t al[4];
            vxo_channel_draw_felt(&ch, al);
            uint32_t half = 1u << (cl - 1);
            Dev tw(half);
            fold_twiddles(vxo_coset_half_odds(cl), false, tw);
            Dev *nx[4];
            for (int c = 0; c < 4; c++) nx[c] = new Dev(half);
            cuda_fold_line_soa(cur[0]->p, cur[1]->p, cur[2]->p, cur[3]->p, tw.p, nx[0]->p, nx[1]->p, nx[2]->p,
                               nx[3]->p, al, half);
            cudaDeviceSynchronize();
            for (int c = 0; c < 4; c++) { delete cur[c]; cur[c] = nx[c]; }
            cl--;
        }
        const uint32_t *fc[4] = {cur[0]->p, cur[1]->p, cur[2]->p, cur[3]->p};
        ftrees.push_back(full_tree(fc, 4, cl));
        const uint32_t *r = ftrees.back().back().data();
        root_only(fc, 4, cl, chk);
        if (memcmp(r, chk, 32)) return 4;
        froots.insert(froots.end(), r, r + 8);
        fvals.push_back({cur[0]->host(), cur[1]->host(), cur[2]->host(), cur[3]->host()});
        vxo_channel_mix_digest(&ch, r);
    }
    for (int c = 0; c < 4; c++) delete cur[c];
    uint32_t last[32];
    for (int i = 0; i < 8; i++) for (int c = 0; c < 4; c++) last[4 * i + c] = fvals.back()[c][i];
    vxo_channel_mix_felts(&ch, last, 8);
    std::vector<uint64_t> qi(nq);
    for (uint32_t j = 0; j < nq; j++) qi[j] = vxo_channel_draw_number(&ch, N);
    // bytes (stark_cli.rs:1092-1123)
    W w;
    w.u(0x4B52414Bu); w.u(1); w.u(log_n); w.u(a); w.u(b);
    w.s(troot, 8); w.s(qroot, 8);
    w.u(nfri); w.s(froots.data(), froots.size());
    w.u(8); w.s(last, 32);
    w.u(nq); for (uint64_t i : qi) w.u((uint32_t)i);
    decom(w, ttree, {&evh}, qi);
    decom(w, qtree, {&qh[0], &qh[1], &qh[2], &qh[3]}, qi);
    w.u(nfri);
    std::vector<uint64_t> fi(nq);
    for (uint32_t j = 0; j < nq; j++) fi[j] = qi[j] >> 1;
    for (uint32_t k = 0; k < nfri; k++) {
        decom(w, ftrees[k], {&fvals[k][0], &fvals[k][1], &fvals[k][2], &fvals[k][3]}, fi);
        for (auto &x : fi) x >>= 1;
    }
    if (cudaGetLastError() != cudaSuccess) return 5;
    size_t bytes = w.w.size() * 4;
    if (bytes > cap) return 6;
    memcpy(out, w.w.data(), bytes);
    *out_len = bytes;
    return 0;
}

// Time the reference's evaluate / interpolate (Forge layer kernels, one
// launch per layer) on 2^log_n points of half_coset(log_n); ms per call.
extern "C" int vxref_ntt_time(uint32_t log_n, uint32_t reps, float *ms_eval, float *ms_interp) {
    uint32_t n = 1u << log_n;
    vxo_coset c = vxo_coset_half_coset(log_n);
    Dev fl(n - 1), fc(n / 2), il(n - 1), ic(n / 2), d(n);
    std::vector<uint32_t> offs, sizes, o2, s2;
    twiddles(c, false, fl, fc, offs, sizes);
    twiddles(c, true, il, ic, o2, s2);
    cudaMemset(d.p, 1, (size_t)n * 4);
    cuda_circle_ntt_evaluate(d.p, fl.p, fc.p, offs.data(), sizes.data(), log_n - 1, n);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (uint32_t r = 0; r < reps; r++) cuda_circle_ntt_evaluate(d.p, fl.p, fc.p, offs.data(), sizes.data(), log_n - 1, n);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms_eval, e0, e1);
    *ms_eval /= reps;
    cudaEventRecord(e0);
    for (uint32_t r = 0; r < reps; r++) cuda_circle_ntt_interpolate(d.p, il.p, ic.p, o2.data(), s2.data(), log_n - 1, n);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms_interp, e0, e1);
    *ms_interp /= reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
