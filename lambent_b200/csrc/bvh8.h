// bvh8.h - compressed 8-wide BVH used by the traversal kernels.
//
// Replaces the driver-side BLAS/TLAS build of the reference (create_blas / create_tlas /
// build_acceleration_structures, examples/cornell_box/src/main.rs:464-563).
//
// Node: 80 bytes = 5 x uint4, child boxes quantized to 8 bits per plane against a per-node
// power-of-two grid (after Ylitie, Karras and Laine, "Efficient Incoherent Ray Traversal on
// GPUs Through Compressed Wide BVHs", HPG 2017):
//   uint4[0] = { px, py, pz (f32 grid origin), ex | ey << 8 | ez << 16 | imask << 24 }
//   uint4[1] = { child_base, leaf_base, meta[0..3], meta[4..7] }
//   uint4[2] = { qlo_x[8], qlo_y[8] }   uint4[3] = { qlo_z[8], qhi_x[8] }   uint4[4] = { qhi_y[8], qhi_z[8] }
// Child box of slot i on axis a: [p_a + qlo_a[i] * 2^(e_a-127), p_a + qhi_a[i] * 2^(e_a-127)],
// padded outward by one grid step so the box test stays conservative under f32 rounding.
// imask bit i: slot i is an internal child; its node index is child_base + popc(imask & ((1<<i)-1)).
// meta[i]: bits 5..7 the slot's hit-mask bits in unary, bits 0..4 their position in the mask.
//   leaf slot: ((1 << count) - 1) << 5 | offset, items leaf_base + offset .. + count - 1 (count 1..3);
//   internal slot: 1 << 5 | (24 + i) (a ray of octant o sets bit 24 + (i ^ o));
//   empty slot: 0 (imask bit clear).
// Slots are assigned so that slot o holds the child a ray of octant o (sign bits x|y<<1|z<<2 of
// its direction) should visit first; traversal visits slot (k ^ octant) for k = 0..7.
#pragma once
#include <cstdint>
#include <vector>

namespace lam {

struct Bvh8Node {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;
    uint32_t child_base, leaf_base;
    uint8_t meta[8];
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
};
static_assert(sizeof(Bvh8Node) == 80, "node must be 80 bytes");

struct Bvh8 {
    std::vector<Bvh8Node> nodes;     // node 0 is the root
    std::vector<uint32_t> leaf_items; // item ids in leaf order
    float lo[3], hi[3];              // exact bounds of all items
};

// boxes: 6 floats per item (lo xyz, hi xyz).  max_leaf in 1..3.  Empty input gives an empty BVH.
void build_bvh8(const float* boxes, uint32_t n, int max_leaf, Bvh8* out);

}  // namespace lam
