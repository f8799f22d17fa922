// fmm_plan.cuh -- interaction offset tables of the uniform-quadtree FMM.
//
// Boxes at level l form a 2^l x 2^l grid of width w_l = w_0 / 2^l.  Two boxes
// at the same level with integer offset (i, j) are WELL SEPARATED when both
//   (theta)  r_1 + r_2 <= theta * d     i.e. (i^2 + j^2) theta^2 >= 2
//   (cutoff) d - r_1 - r_2 >= cutoff   i.e. (sqrt(i^2 + j^2) - sqrt 2) w_l >= cutoff
// hold (r = half diagonal, d = centre distance).  These are the two checks of
// the reference FMM's connectivity (theta = 1/2, THETACUTOFFCHECK:
// src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm.cpp:1735-1835): the Gaussian core
// must be negligible for every far pair.  Because the tree is uniform the
// lists depend only on the offset, not on the box, and are built once per plan:
//
//   near[l]         offsets that are not well separated, closed upwards so
//                   that the parent of every near box is near at level l-1;
//   far[l][pos]     M2L list of a box at child position pos: children of the
//                   parent's near boxes that are not near the box itself
//                   (at the leaf level pos = px + Bp*py, (px, py) = leaf
//                   coordinates mod Bp, Bp = max(2^kb, 2));
//   p2p             leaf offsets, relative to the origin leaf of a P2P block
//                   (2^kb x 2^kb leaves), whose particles every target of the
//                   block interacts with directly (union of the members' near
//                   sets); the leaf-level far lists exclude exactly this set,
//                   so every (target leaf, source leaf) pair is covered once.
#pragma once
#include <stdint.h>

#include <vector>

namespace pf {
namespace fmm {

struct Off {
    int i, j;
    bool operator<(const Off &o) const { return i < o.i || (i == o.i && j < o.j); }
    bool operator==(const Off &o) const { return i == o.i && j == o.j; }
};

struct Tables {
    int L = 0;                                     // leaf level
    int kb = 1;                                    // P2P block = 2^kb x 2^kb leaves
    double w0 = 1.0, cutoff = 0.0, theta = 0.5;
    std::vector<std::vector<Off>> near;            // [l]
    std::vector<std::vector<std::vector<Off>>> far;  // [l][pos]
    std::vector<Off> p2p;                          // block-relative leaf offsets
};

// Build every table for a tree with leaf level L.
void build_tables(int L, int kb, double w0, double cutoff, double theta, Tables &t);

// What the tables depend on: for each level l = 0..L, the smallest integer
// s2 = i^2 + j^2 whose offsets are well separated at that level (both checks
// are monotone in s2), or 2 (2^l - 1)^2 + 1 when none is.  Two (w0, cutoff)
// pairs with the same key build the same tables, so plans are keyed by it
// rather than by the exact cutoff / width ratio of a moving blob set.
void separation_key(int L, double w0, double cutoff, double theta, std::vector<int64_t> &key);

// Flattened form (int32), shared with pf_fmm_lists():
//   L, kb, then for l = 0..L: n, (i, j) * n;
//   then for l = 1..L: npos, for each pos: n, (i, j) * n;
//   then n_p2p, (i, j) * n_p2p.
void flatten(const Tables &t, std::vector<int32_t> &out);

}  // namespace fmm
}  // namespace pf
