// Device-resident Fibonacci prover: layout of the proof bytes and the
// per-size / per-proof device state.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "vx_merkle.cuh"

namespace vx {

// Word offsets of every field of the proof in the reference's "KRAK" v1
// layout (stark_cli.rs:1092-1123): header, roots, FRI roots, last layer,
// query indices, then the trace, quotient and FRI decommitments.
struct DecomLayout {
    uint64_t n, vals, svals, paths, spaths;
    uint32_t width, depth;
};
struct ProofLayout {
    uint32_t log_n, blowup, le, nfri, nq;
    uint64_t words;
    uint64_t magic, troot, qroot, nfri_w, froots, nlast, last, nq_w, qidx, nfd;
    DecomLayout trace, quot, fri[32];
};
void proof_layout(uint32_t log_n, uint32_t blowup, uint32_t nq, ProofLayout *L);


// Read-only tables for one (log_n, blowup) on one device.
struct SizeTables {
    int device;
    uint32_t log_n, blowup, le;
    uint32_t *itw_line, *itw_circle;  // inverse tables of half_coset(log_n)
    uint32_t *ftw_line, *ftw_circle;  // forward tables of the eval domain
    uint32_t *fold_circle;            // circle-fold twiddles of the eval domain
    uint32_t *fold_line;              // line-fold twiddles, half_odds(l) for l = le-1 .. 4
    uint64_t fold_line_off[32];       // offset of half_odds(l)'s table, indexed by l
    uint32_t itw_off[32], ftw_off[32];
    void *block;                      // single allocation backing the tables
};

// Per in-flight proof state.
struct ProofSlot {
    SizeTables *tw;
    ProofLayout L;
    uint32_t *coeffs, *eval;
    uint32_t *fri[32][4];          // FRI layer k, 4 SoA columns of 2^(le-1-k)
    TreeLevels trace_lv, quot_lv, fri_lv[32];
    DevChannel *chan;
    uint32_t *alpha_q;             // 4 words
    uint32_t *alpha_f;             // 4 words per FRI fold
    uint32_t *qidx;                // n_queries words
    uint32_t *proof;               // device proof, L.words words
    const uint32_t *inputs;        // device (a, b) for captured graphs; null = kernel arguments
    void *block;                   // single allocation backing the above
    size_t block_bytes;
};

}  // namespace vx

struct vx_prover;
namespace vx {
// One whole proof as a CUDA graph: (a, b) read from pinned_ab, the proof
// bytes copied to pinned_out followed by the 4-byte transcript status word
// (pinned_out holds prover_proof_bytes + 4 bytes).
int prover_capture_graph(vx_prover *p, cudaStream_t st, uint32_t *dev_ab, const uint32_t *pinned_ab,
                         void *pinned_out, cudaGraphExec_t *exec);
// The same proof split into two graphs at stage `split`: head (inputs in,
// stages before split) and tail (the rest, proof bytes and status word out).
// At split 6 (the line folds) the head also takes the FRI layers whose trees
// are deeper than 16; the tail starts with the first smaller layer.
int prover_capture_graph_split(vx_prover *p, cudaStream_t st, uint32_t *dev_ab, const uint32_t *pinned_ab,
                               void *pinned_out, uint32_t split, cudaGraphExec_t *head, cudaGraphExec_t *tail);
uint32_t prover_log_n(const vx_prover *p);
void prover_footprint(uint32_t log_n, uint32_t blowup, uint32_t nq, size_t *slot_b, size_t *tab_b);
size_t prover_proof_bytes(const vx_prover *p);
const uint32_t *prover_chan_err(const vx_prover *p);
// Frees the forge batch launchers' per-device column-pointer arrays.
void forge_cols_release();
}  // namespace vx
