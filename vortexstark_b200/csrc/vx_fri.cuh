// FRI fold fused with the commitment of the folded layer.
#pragma once
#include <cstdint>

#include "vx_field.cuh"

namespace vx {

// Leaf source for a tree over a folded SoA4 QM31 layer: output j pairs
// f0 = in[2j] and f1 = in[2j + 1] (fri.cu:58-126),
//   out[j] = (f0 + f1) + alpha * ((f0 - f1) * tw[j]),
// stored to the output layer and hashed as its 4-word leaf.  The circle fold
// into a pre-zeroed line (fri.cu:92-126) is the same formula; line and
// circle folds differ only in their twiddles.
struct LeafFold {
    const uint32_t *i0, *i1, *i2, *i3;
    const uint32_t *tw;
    const uint32_t *alpha_ptr;
    uint32_t *o0, *o1, *o2, *o3;
    qmat am;  // multiplication by the fold challenge
    __device__ __forceinline__ void init() { am = qmat_of(qm31{{alpha_ptr[0], alpha_ptr[1], alpha_ptr[2], alpha_ptr[3]}}); }
    __device__ __forceinline__ uint32_t load(uint64_t j, uint32_t m[16]) const {
        uint2 a0 = __ldg((const uint2 *)i0 + j), a1 = __ldg((const uint2 *)i1 + j);
        uint2 a2 = __ldg((const uint2 *)i2 + j), a3 = __ldg((const uint2 *)i3 + j);
        qm31 f0{{a0.x, a1.x, a2.x, a3.x}}, f1{{a0.y, a1.y, a2.y, a3.y}};
        qm31 r = qadd(qadd(f0, f1), qmul_mat(am, qmulm(qsub(f0, f1), __ldg(tw + j))));
        o0[j] = r.v[0]; o1[j] = r.v[1]; o2[j] = r.v[2]; o3[j] = r.v[3];
        m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
        return 16u;
    }
};

}  // namespace vx
