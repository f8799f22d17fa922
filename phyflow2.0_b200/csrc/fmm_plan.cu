// fmm_plan.cu -- host construction of the FMM offset tables (see fmm_plan.cuh).
#include <algorithm>
#include <cmath>
#include <set>

#include "fmm_plan.cuh"
#include "pf_common.cuh"

namespace pf {
namespace fmm {

static bool separated_s2(int64_t k, double w, double cutoff, double theta) {
    const double s2 = (double)k;
    const bool sep_theta = s2 * (theta * theta) >= 2.0;
    const bool sep_cut = (std::sqrt(s2) - std::sqrt(2.0)) * w >= cutoff;
    return sep_theta && sep_cut;
}

static bool well_separated(int i, int j, double w, double cutoff, double theta) {
    return separated_s2((int64_t)i * i + (int64_t)j * j, w, cutoff, theta);
}

void separation_key(int L, double w0, double cutoff, double theta, std::vector<int64_t> &key) {
    key.assign(L + 1, 0);
    for (int l = 0; l <= L; ++l) {
        const int64_t ext = ((int64_t)1 << l) - 1;
        const double w = std::ldexp(w0, -l);
        int64_t lo = 0, hi = 2 * ext * ext + 1;  // answer in [lo, hi]; hi: none separated
        while (lo < hi) {
            const int64_t mid = lo + (hi - lo) / 2;
            if (separated_s2(mid, w, cutoff, theta))
                hi = mid;
            else
                lo = mid + 1;
        }
        key[l] = lo;
    }
}

static int floordiv2(int a) { return (a >= 0) ? a / 2 : -((-a + 1) / 2); }

void build_tables(int L, int kb, double w0, double cutoff, double theta, Tables &t) {
    t.L = L;
    t.kb = kb;
    t.w0 = w0;
    t.cutoff = cutoff;
    t.theta = theta;
    t.near.assign(L + 1, {});
    t.far.assign(L + 1, {});
    std::vector<std::set<Off>> nset(L + 1);
    for (int l = 0; l <= L; ++l) {
        const int ext = (1 << l) - 1;
        const double w = std::ldexp(w0, -l);
        const double rmax = std::max(std::sqrt(2.0) / theta, cutoff / w + std::sqrt(2.0));
        const int R = (int)std::min<double>(ext, std::ceil(rmax) + 1.0);
        for (int i = -R; i <= R; ++i)
            for (int j = -R; j <= R; ++j)
                if (!well_separated(i, j, w, cutoff, theta)) nset[l].insert({i, j});
    }
    // P2P block union at the leaf level, and its per-position near sets
    const int B = 1 << kb;
    const int extL = (1 << L) - 1;
    std::set<Off> q;
    for (int cx = 0; cx < B; ++cx)
        for (int cy = 0; cy < B; ++cy)
            for (const Off &o : nset[L]) {
                Off s{o.i + cx, o.j + cy};
                q.insert(s);
            }
    t.p2p.assign(q.begin(), q.end());
    std::vector<std::set<Off>> nleaf(B * B);  // N'_L(cb), cb = cx + B*cy
    for (int cx = 0; cx < B; ++cx)
        for (int cy = 0; cy < B; ++cy) {
            auto &s = nleaf[cx + B * cy];
            for (const Off &a : q) {
                Off o{a.i - cx, a.j - cy};
                if (std::abs(o.i) <= extL && std::abs(o.j) <= extL) s.insert(o);
            }
        }
    // closure: parents of near boxes are near one level up
    if (L >= 1) {
        for (int cx = 0; cx < B; ++cx)
            for (int cy = 0; cy < B; ++cy) {
                const int c0 = cx & 1, c1 = cy & 1;
                for (const Off &o : nleaf[cx + B * cy]) {
                    Off p{floordiv2(c0 + o.i), floordiv2(c1 + o.j)};
                    const int ext = (1 << (L - 1)) - 1;
                    if (std::abs(p.i) <= ext && std::abs(p.j) <= ext) nset[L - 1].insert(p);
                }
            }
        for (int l = L - 1; l >= 1; --l) {
            const int ext = (1 << (l - 1)) - 1;
            std::vector<Off> cur(nset[l].begin(), nset[l].end());
            for (int c0 = 0; c0 < 2; ++c0)
                for (int c1 = 0; c1 < 2; ++c1)
                    for (const Off &o : cur) {
                        Off p{floordiv2(c0 + o.i), floordiv2(c1 + o.j)};
                        if (std::abs(p.i) <= ext && std::abs(p.j) <= ext) nset[l - 1].insert(p);
                    }
        }
    }
    for (int l = 0; l <= L; ++l) t.near[l].assign(nset[l].begin(), nset[l].end());
    // far (M2L) lists
    // leaf-level positions index a Bp x Bp block, Bp = max(B, 2), so that they
    // determine both the child position (for the candidates) and the position
    // in the P2P block (for the near set)
    const int Bp = B > 2 ? B : 2;
    for (int l = 1; l <= L; ++l) {
        const int ext = (1 << l) - 1;
        const int npos = (l == L) ? Bp * Bp : 4;
        t.far[l].assign(npos, {});
        for (int pos = 0; pos < npos; ++pos) {
            int c0, c1;
            const std::set<Off> *own;
            if (l == L) {
                const int px = pos % Bp, py = pos / Bp;
                c0 = px & 1;
                c1 = py & 1;
                own = &nleaf[(px % B) + B * (py % B)];
            } else {
                c0 = pos & 1;
                c1 = (pos >> 1) & 1;
                own = &nset[l];
            }
            std::set<Off> f;
            for (const Off &O : nset[l - 1])
                for (int d0 = 0; d0 < 2; ++d0)
                    for (int d1 = 0; d1 < 2; ++d1) {
                        Off o{2 * O.i + d0 - c0, 2 * O.j + d1 - c1};
                        if (std::abs(o.i) > ext || std::abs(o.j) > ext) continue;
                        if (own->count(o)) continue;
                        f.insert(o);
                    }
            t.far[l][pos].assign(f.begin(), f.end());
        }
    }
}

void flatten(const Tables &t, std::vector<int32_t> &out) {
    out.clear();
    out.push_back(t.L);
    out.push_back(t.kb);
    for (int l = 0; l <= t.L; ++l) {
        out.push_back((int32_t)t.near[l].size());
        for (const Off &o : t.near[l]) {
            out.push_back(o.i);
            out.push_back(o.j);
        }
    }
    for (int l = 1; l <= t.L; ++l) {
        out.push_back((int32_t)t.far[l].size());
        for (const auto &f : t.far[l]) {
            out.push_back((int32_t)f.size());
            for (const Off &o : f) {
                out.push_back(o.i);
                out.push_back(o.j);
            }
        }
    }
    out.push_back((int32_t)t.p2p.size());
    for (const Off &o : t.p2p) {
        out.push_back(o.i);
        out.push_back(o.j);
    }
}

}  // namespace fmm
}  // namespace pf

extern "C" pf_status pf_fmm_lists(int leaf_level, int block_level_drop, double root_width,
                                  double cutoff, double theta, int32_t *buf, int64_t capacity,
                                  int64_t *needed) {
    pf::clear_error();
    PF_CHECK_ARG(leaf_level >= 1 && leaf_level <= 16, "pf_fmm_lists: leaf level %d outside [1, 16]",
                 leaf_level);
    PF_CHECK_ARG(block_level_drop >= 0 && block_level_drop <= 3 && block_level_drop <= leaf_level,
                 "pf_fmm_lists: block level drop %d outside [0, min(3, L)]", block_level_drop);
    PF_CHECK_ARG(root_width > 0.0 && std::isfinite(root_width), "pf_fmm_lists: bad root width");
    PF_CHECK_ARG(cutoff >= 0.0 && std::isfinite(cutoff), "pf_fmm_lists: bad cutoff");
    PF_CHECK_ARG(theta > 0.0 && theta < 1.0, "pf_fmm_lists: theta must be in (0, 1)");
    PF_CHECK_ARG(needed != nullptr, "pf_fmm_lists: needed is NULL");
    pf::fmm::Tables t;
    pf::fmm::build_tables(leaf_level, block_level_drop, root_width, cutoff, theta, t);
    std::vector<int32_t> flat;
    pf::fmm::flatten(t, flat);
    *needed = (int64_t)flat.size();
    if ((int64_t)flat.size() > capacity || !buf) {
        pf::set_error("pf_fmm_lists: needs %lld ints", (long long)flat.size());
        return PF_ERR_CAPACITY;
    }
    std::copy(flat.begin(), flat.end(), buf);
    return PF_OK;
}
