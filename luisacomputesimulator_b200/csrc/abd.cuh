// abd.cuh -- affine bodies (the reference's ABD: Solver/SimulationSolver/newton_solver.cpp:1176-1414,
// Solver/SimulationCore/affine_position.h, collision_data.h:198-268, narrow_phase.cpp:2598-2676).
//
// A body's 12 DOFs q = [p, a0, a1, a2] move its vertices by x = p + x_bar.x a0 + x_bar.y a1 + x_bar.z a2
// (J = [I, x_bar.x I, x_bar.y I, x_bar.z I]).  Here the four 3-vectors of q live in four "DOF slot"
// vertex records of the body's scene (vertex ids body_dof[b] .. body_dof[b] + 3), so the Newton system's
// rows stay vertex ids: slot rows carry q, its increment and its velocity through the same per-vertex
// kernels as cloth vertices, while the rows of the body's mesh vertices are inert (identity diagonal,
// zero right-hand side) and their positions follow q.  Slots take no part in contact queries (their
// d_hat is negative).
#pragma once
#include "lcs_common.cuh"
#include "lcs_geom.cuh"

namespace lcs {

// per-vertex body ids (kInvalid: soft), body-frame rest positions, first DOF slot per body
struct AbdView {
    const uint32_t* body;
    const float4* model_x;
    const uint32_t* body_dof;
};

// p + x_bar.x a0 + x_bar.y a1 + x_bar.z a2 (AffineBodyDynamics, A * rest_x + p)
__device__ __forceinline__ v3 affine_apply(v3 p, v3 a0, v3 a1, v3 a2, float4 m)
{
    return mk3(((a0.x * m.x + a1.x * m.y) + a2.x * m.z) + p.x, ((a0.y * m.x + a1.y * m.y) + a2.y * m.z) + p.y,
               ((a0.z * m.x + a1.z * m.y) + a2.z * m.z) + p.z);
}

// The generalised DOFs of a contact pair (get_active_indices, collision_data.h:198-268): each side (VF:
// vertex 0 | face 1..3; EE: edge 0,1 | edge 2,3) is either soft -- its vertices with their weights -- or
// rigid -- its body's four DOF slots with weights sum_i w_i (1, x_bar_i) (add_to_rigid_body,
// narrow_phase.cpp:2612-2629).  A side's body is that of vertex 0 (left) or vertex 2 (right).
__device__ __forceinline__ int pair_dofs(const PairView& P, const AbdView& a, uint32_t dof[8], float gw[8])
{
    const int split = P.type == 1 ? 1 : 2;
    int n = 0;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const int s0 = side ? split : 0, s1 = side ? 4 : split;
        const uint32_t b = a.body[P.v[side ? 2 : 0]];
        if (b == kInvalid) {
            for (int i = s0; i < s1; ++i) {
                dof[n] = P.v[i];
                gw[n] = P.w[i];
                ++n;
            }
        } else {
            float w0 = 0.0f, w1 = 0.0f, w2 = 0.0f, w3 = 0.0f;
            for (int i = s0; i < s1; ++i) {
                const float4 m = a.model_x[P.v[i]];
                w0 += P.w[i];
                w1 += P.w[i] * m.x;
                w2 += P.w[i] * m.y;
                w3 += P.w[i] * m.z;
            }
            const uint32_t d0 = a.body_dof[b];
            dof[n] = d0; gw[n] = w0; ++n;
            dof[n] = d0 + 1; gw[n] = w1; ++n;
            dof[n] = d0 + 2; gw[n] = w2; ++n;
            dof[n] = d0 + 3; gw[n] = w3; ++n;
        }
    }
    return n;
}

}  // namespace lcs
