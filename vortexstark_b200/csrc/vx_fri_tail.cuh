// A run of FRI fold layers, each committed with its transcript step.
//
// Every FRI path here folds layer k-1 into layer k, commits layer k as a
// 4-word-leaf Blake2s tree and mixes its root before drawing the next
// challenge (prover.rs:860-926 with fri.rs:163-224).  Large layers go through
// tree_build with a LeafFold source.  The small layers at the end of the run
// are latency-bound: each is a chain of about depth + 3 dependent
// compressions, and one launch per layer adds a launch gap, a prologue and a
// global round trip of the folded values.  fold_layers therefore runs the
// consecutive layers of at most 2^kTailMaxLog values in one single-block
// launch, with the folded values and digests in shared memory.  Its stored
// tree levels, layer values, proof roots, transcript state and challenges are
// the words the per-layer launches write.
#pragma once
#include <cstdint>

#include "vx_merkle.cuh"

namespace vx {

constexpr uint32_t kTailMaxLog = 10;   // layers of at most 2^10 values go to the tail kernel
constexpr uint32_t kTailMaxLayers = 12;

// One fold layer: out[j] = (f0 + f1) + alpha * ((f0 - f1) * tw[j]) with
// f0 = in[2j], f1 = in[2j + 1] for j < 2^depth (lv's depth).
struct FoldLayer {
    const uint32_t *in[4];   // 2^(depth+1) values (SoA QM31)
    const uint32_t *tw;      // 2^depth twiddles
    const uint32_t *alpha;   // the layer's challenge (4 words, device)
    uint32_t *out[4];        // 2^depth values
    TreeLevels lv;           // the layer's tree
    ChanStep cs;             // root into the proof, mix, next challenge
};

// Enqueue layers [0, n) in order on `st`; layers[k].in must be
// layers[k-1].out for the tail to fuse them.  *launches grows by the kernel
// launches enqueued.
cudaError_t fold_layers(const FoldLayer *layers, uint32_t n, cudaStream_t st, uint32_t *launches);

}  // namespace vx
