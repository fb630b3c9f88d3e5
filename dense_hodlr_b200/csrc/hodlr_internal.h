// Internal structures shared by the kernels and the host orchestration.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kfun.h"

// Where a matrix entry comes from: a kernel of point coordinates, or a
// dense column-major matrix resident in HBM.
struct EntrySrc {
  const double* pts;  // SoA coordinates, pts[d * ld + i]
  const double* A;    // dense input, A[i + j * ld]
  int64_t ld;         // = n
  hx_kparams kp;
  int dense;
  // forest of independent systems: kernel of system psys[i] (null for one system)
  const hx_kparams* kps;
  const int* psys;
};

// ----------------------------------------------------------------- ACA
enum {
  ACA_RUNNING = 0,   // loop in progress (or not started)
  ACA_POST = 1,      // loop finished, post-processing pending
  ACA_DONE = 2,      // W, V and rank final
  ACA_NEED_CAP = 3,  // loop paused: more columns of W/V are needed
  ACA_ERROR = 4,
  ACA_NEED_CAP_POST = 5,  // loop done; the full-rank form needs more columns
};

// One off-diagonal block.  W and V point at the block's first row inside the
// level arenas (leading dimension = N), so W(i,l) = W[i + l*N] for the block's
// local row i, and V(j,l) = V[j + l*N] for its local column j.
struct AcaState;

struct AcaBlock {
  AcaState* st;       // loop state of this block
  double* W;
  double* V;
  unsigned char* cR;  // chosen rows, local index
  unsigned char* cC;  // chosen columns, local index
  int* prow;          // pivot row of step t, local index
  int* pcol;          // pivot column of step t
  int r0, c0, m, n;
  int kcap;           // columns available in W and V
  int level;
  int g0, G;          // with a CTA table: first CTA of this block's group, group size
  int minRank, maxRank;  // the node's rank bounds for this block (-1: none)
};

// Loop state of one block; lets a paused block resume where it stopped.
struct AcaState {
  double frob2, eps, margin;
  double swp, svp;  // |w_{k-1}|^2, |v_{k-1}|^2 while epsilon_{k-1} is pending
  int k, cur, status, iters, rank, near;
  int pending;      // 1: epsilon of step k-1 not evaluated yet
  int pad;
};

struct AcaLaunch {
  const AcaBlock* blocks;
  int nblocks;
  int G;                 // CTAs per block
  int64_t ld;            // N
  double tol, minPivot;
  int kcap_max;          // largest kcap among the launch's blocks (shared memory rows)
  double* part;          // per-CTA partials, part_stride doubles each
  int64_t part_stride;
  unsigned* bar;         // per-block barrier counters (zeroed before launch)
  unsigned* err;         // device error word
  EntrySrc src;
  const int* cta_block;  // CTA -> block (groups of uneven size, AcaBlock::g0/G), or null
  int ncta;              // CTAs of the launch when cta_block is set
  double* dotg;          // per-CTA per-warp dot partials in global memory (large ranks), or null
  int64_t dotg_stride;   // doubles per CTA in dotg (NT/32 * kcap_max)
  int ring;              // 1: panel slices streamed by per-warp bulk-copy rings (512
                         //    threads, even ld)
  int ring_stages;       // stages of each warp's ring (aca_ring_stages(kcap_max))
  int narrow;            // 1 (256 threads, no ring): 2 elements per thread, 512-row chunks
  unsigned spin_limit;   // polls of a group barrier before it gives up (DEV_ERR_TIMEOUT)
  unsigned bar_extra;    // arrivals a group barrier waits for beyond its G CTAs (0; 1 makes
                         // every barrier unreachable, to exercise the timeout path)
  int ring_tile;         // 1 (with ring): each ring tile is one 2D tensor copy through
                         // map_w / map_v instead of one bulk copy per column
  // 2D maps over the level's W and V arenas (rows: N, columns: the level's
  // kcap, row stride ld), box WR_ROWS rows x WR_BC columns; set when ring_tile
  alignas(64) CUtensorMap map_w;
  alignas(64) CUtensorMap map_v;
};
