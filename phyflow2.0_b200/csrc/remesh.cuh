// remesh.cuh -- the M4' / Tutty remesh core shared by the remesh entry points,
// the batched step and the no-allocation variant.
#pragma once
#include "popctl.cuh"

namespace pf {

constexpr int REMESH_M4 = 0;     // M4' weights with the Wee coefficient c
constexpr int REMESH_TUTTY = 1;  // Tutty weights with c = hNu

// Per-call state on the device, zeroed (with the base-cell counts behind it)
// by one memset at the start of every call.
struct RmHead {
    // window extent as max(ix + IDX_OFF) and max(IDX_OFF - ix) over the finite
    // blobs, so that zero is the neutral start (0: no finite blob)
    int32_t xhi, xlo, yhi, ylo;
    // 1: NaN/Inf coordinate, 2: lattice index beyond +-2^30, 4: blob outside
    // the window (skipped), 8: window beyond the scratch capacity or the dense
    // limit (nothing done)
    int32_t bad;
    uint32_t ticket;  // CTAs of the extent pass that finished
    int32_t total;    // output count
    int32_t big_n;    // cells of more than SEG_SMALL blobs listed for the segment sort
    int32_t ixmin, iymin, nbx, nby;  // the window (valid when ok)
    int32_t ok;
    uint32_t ticket_in, ticket_out;  // CTAs of k_rm_place / k_rm_tile that finished
    int32_t pad;
    int64_t ncell;  // (nbx + 3) (nby + 3) when ok, else 0
    int64_t pad2;
    // FP64 moments {sum g, sum g x, sum g y, sum |g|} of the blobs placed in
    // the window and of the new blobs (M4' / Tutty emit path), each summed
    // in a fixed order
    double mom[8];
    // compressed window (sparse blob sets): the sorted lattice rows / columns
    // that window rows / columns stand for; null for a dense window
    const int32_t *rows, *cols;
};
static_assert(sizeof(RmHead) == 160, "RmHead layout");
constexpr int32_t RM_IDX_OFF = (1 << 30) + 1;

// Where the base-cell window comes from, and the scratch capacity.
struct RmWindow {
    bool from_blobs;        // computed on the device from the blobs (extent pass)
    int32_t ixmin, iymin;   // else given: base cells [ixmin, ixmin + nbx) x [iymin, ...)
    int64_t nbx, nby;
    int64_t cap_base;       // base cells the scratch holds (>= nbx nby when given)
    int64_t cap_cell;       // output cells the scratch holds (>= (nbx + 3)(nby + 3))
    int64_t cell_limit;     // largest admissible window in base cells (from_blobs)
    // compressed window (given windows only): DEVICE sorted lattice rows[nbx]
    // and cols[nby] that contain every blob's base row xl with xl+1..xl+3
    // (and the same for columns); window row bx stands for lattice row
    // rows[bx].  Null: the dense window above.
    const int32_t *rows = nullptr, *cols = nullptr;
};

// Scratch bytes of remesh_core for n blobs and the given capacities;
// `cells_mode` adds the per-cell value and flag arrays of the population-
// control path.  Capacities must be below 2^31 (callers check).
size_t remesh_scratch_bytes(int64_t n, int64_t cap_base, int64_t cap_cell, bool cells_mode);

// Enqueue the remesh: no host synchronisation, nothing allocated.  *total
// receives the output count (0 when the window was rejected), *bad is OR-ed
// with the head's flags (the caller zeroes it).  head_out (may be null)
// receives the device address of this call's RmHead (valid until the scratch
// is reused).  pc: population control of the cells before they are emitted.
pf_status remesh_core(Bump &sc, int64_t n, const double *x, const double *y, const double *g,
                      double h, double xb0, double yb0, double c, const RmWindow &win,
                      int64_t capacity, double *xo, double *yo, double *go, int64_t *ixo,
                      int64_t *iyo, int32_t *total, int32_t *bad, cudaStream_t st, int num_sms,
                      const PopCtlArgs *pc = nullptr, int kernel = REMESH_M4,
                      RmHead **head_out = nullptr);

// Write a call's output count, status word (RmHead::bad), window
// {ixmin, iymin, nbx, nby} and the 8 moments (each pointer may be null) to
// device memory.
pf_status remesh_finish(const RmHead *hd, int64_t *n_out_dev, int32_t *status_dev,
                        int64_t *window_dev, double *moments_dev, cudaStream_t st);

// Base-cell window of a blob set whose lattice left indices span
// [ixmin, ixmax] x [iymin, iymax], decoded from a head.
__host__ __device__ inline bool rm_head_window(const RmHead &h, int64_t &ixmin, int64_t &iymin, int64_t &nbx,
                           int64_t &nby) {
    if (h.xhi == 0 || h.yhi == 0) return false;
    ixmin = (int64_t)RM_IDX_OFF - h.xlo;
    iymin = (int64_t)RM_IDX_OFF - h.ylo;
    nbx = ((int64_t)h.xhi - RM_IDX_OFF) - ixmin + 1;
    nby = ((int64_t)h.yhi - RM_IDX_OFF) - iymin + 1;
    return true;
}

}  // namespace pf
