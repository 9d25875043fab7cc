// Kernel argument blocks shared by the CUDA kernels and the C++ host.
#pragma once
#include <cstdint>

namespace zb {

enum Metric { M_SSD = 0, M_SAD = 1, M_ZSSD = 2, M_ZSAD = 3, M_SSD_NORM = 4 };

// Block matching of one plane entry.  Reference blocks sit at
// x = min(bs*kx, w-8), y = min(bs*ky, h-8) (vszipcu src/bm3d.cu:585-595).
struct MatchArgs {
    const float *frames;   // matching plane of window frame t at frames + t*fstride
    long long fstride;
    int w, h, pitch;
    int bs, range;
    int radius, ps_num, ps_range;
    int nbx, nby;          // reference blocks per row / column
    int nbx_al;            // blocks whose x = bs*kx needs no clamp
    int tile_pitch;        // shared tile row pitch in floats (tiled kernel)
    int chunks;            // ceil((2*range+1)/4)
    int2 *list;            // [nby*nbx][8]: (x, y | z << 24)
    float *errs;           // [nby*nbx][8]: distances of the spatial list (radius > 0)
    int self_incl;         // 1: insert the block itself here (radius 0)
    int gen_mode;          // generic kernel: 0 = every block, 2 = the blocks listed in tc_ws
                           // (fallbacks of the tensor-core form)
    // Tensor-core form (zb3d_match_tc.cu).  tc_ws: [0] number of listed fallback
    // blocks, [kTcWsList..] their block indices.  tc_stats (optional, accumulated):
    // [0] tiles, [1] blocks, [2] re-ranked candidates, [3] fallback blocks.
    int *tc_ws;
    unsigned long long *tc_stats;
    float *tc_dbg;         // optional: pass-1 distances of tile (0, 0), [128][tiles flat candidates]
    unsigned long long *tc_prof;  // optional: per tile [16]: clock64 phase marks [0..7], mbarrier
                                  // polls of the block and issuer warps [8], [10], TMEM load cycles
                                  // and count [11], [13], pass-1 / pass-2 / done-wait cycles [12], [14], [15]; then for tile (1, 1) a per-job trace
                                  // [job][3] (issued, completion seen, slot freed), at most 64 jobs
};

constexpr int kTcWsList = 8;

// Collaborative filtering + aggregation of one plane entry.
struct FilterArgs {
    const float *src;                 // [clips][planes][tw][h][pitch]
    long long clip_stride, plane_stride, frame_stride;
    int w, h, pitch;
    int nplanes, chroma;
    const int2 *list;                 // [nblocks][8]
    int nblocks;
    float sigma[3];                   // already scaled (hard or Wiener factor)
    float extractor;                  // 2^extractor_exp, or 0
    unsigned long long *num;          // [planes][tw][h][pitch]  fixed point, 2^32 = 1.0
    unsigned long long *den;          // [planes][tw][h][pitch]  weights at patch origins
    long long acc_plane_stride, acc_frame_stride;
};

// One plane entry of a batch (zb3d_process_batch): its matching and filtering arguments
// (own list and accumulators) and its place in the batch's work list.  Items are numbered
// match tiles first (all entries), then filter chunks (all entries).
struct BatchEntry {
    MatchArgs m;                      // tile_pitch, chunks and self_incl set; bs 4 or 8
    FilterArgs f;
    int tiles_x;                      // match tiles per tile row (31 or 16 block columns each)
    int match_items;                  // match tiles (kBatchMatchRows block rows each)
    int filter_items;                 // filter chunks (kBatchGroups groups each)
    long long first_match, first_filter;  // first item number of each kind
};

struct BatchArgs {
    const BatchEntry *entries;
    int nentries;
    long long match_total, items_total;   // match items, all items
    unsigned long long *next;         // next item to take (starts at 0)
    unsigned *match_done;             // [nentries] match tiles finished
    int *status;                      // 0, or 1 when a filter chunk gave up waiting for its matching
    unsigned wait_polls;              // polls (about 0.1 us apart) before a wait gives up
    int unsatisfiable;                // testing: entry 0's chunks wait for one tile more than it has
};

constexpr int kBatchGroups = 128;     // groups per filter chunk
constexpr int kBatchMatchRows = 8;    // block rows (warps) per match tile

// Fixed-point scale of the accumulators: value * 2^32 held in a signed 64-bit sum.
constexpr float kFixScale = 4294967296.0f;
constexpr float kFixInv = 2.3283064365386962890625e-10f;

}  // namespace zb
