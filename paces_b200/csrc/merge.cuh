// Structured k-way merge: basis expansion, sort and dedup without a general sort.
//
// Reference behaviour (paces/core/hamiltonian.py:550-577 enlarge_basis_set,
// :383-492 generate_mel, paces/aux/helpers.py:63-75 cupy_unique): collect the
// basis and every image of every basis state under the off-diagonal terms, lexsort
// the rows and drop duplicates.
//
// B200 design: keys carry only the phonon words; the exciton position is the block.
// For a sorted basis X the candidates of output block p are five runs, each already
// sorted because every Holstein term maps a sorted block monotonically:
//   SELF       X_p                      (the basis itself)
//   FROM_LEFT  X_{p-1}                  (right hops land in block p, phonon words unchanged)
//   FROM_RIGHT X_{p+1}                  (left hops)
//   UP         X_p with n_p + 1         (b^dagger at the exciton site; ceiling n_p = maxd-1 is a hole)
//   DOWN       X_p with n_p - 1         (b at the exciton site; floor n_p = 0 is a hole)
// Lattices with more hopping channels (geo_dim > 1, hopping2) run further passes whose
// runs are the previous output and two more channels' images (RunKind, merge_passes).
// An expansion may also take a keep mask over the images (the learned proposal): a
// dropped image keeps its key and sorts like a ceiling hole, so it is never emitted.
// A hole keeps a placeholder key that preserves the run's order (DOWN: fields after p
// cleared; UP: all bits below field p set) and a flag that sorts it before (DOWN) or
// after (UP) real keys with the same words, so holes never produce output.
//
// The merge is tiled with splitters: every `stride`-th element of every run is ranked
// against all runs (binary search), splitters are put in merged order, and every
// `group` consecutive splitters bound one tile of at most (group + 5) * stride elements.
// A tile is merged in shared memory (a pairwise merge tree with merge-path splits),
// duplicates are flagged against the merged predecessor, and output offsets come from a
// decoupled look-back over tiles taken in ticket order.  Every input element learns the
// index of its key in the output, which gives the H neighbour table without any lookup.
#pragma once

#include "common.cuh"

namespace paces {

struct MergeWs {
    int* run_lo;     // [L*kRuns] first source index in X of each run
    int* run_len;    // [L*kRuns]
    int* split_off;  // [L*kRuns + 1] prefix of splitter counts
    int* tile_off;   // [L + 1] prefix of tile counts
    int* counters;   // [0] splitters [1] tiles [2] tile ticket [3] ceiling holes [4] output count
                     // [5] tile blocks done
    int* split_co;   // [split_cap * kRuns]
    int* split_rank; // [split_cap]
    int* ord_co;     // [split_cap * kRuns]
    unsigned long long* tile_state;  // [tile_cap] look-back words
    unsigned char* tile_desc;        // [tile_cap] tile descriptors (merge_desc_bytes each)
    int split_cap;
    int tile_cap;
    // optional candidate filter (expansion only): keep[j * keep_cap + src] == 0 drops the
    // image of source element src under run j (j = 1..4); dropped images sort like
    // ceiling holes (after real elements with the same key) and are never emitted
    const uint8_t* keep;
    int64_t keep_cap;
    // what each run is (run 0 is always the self run): see RunKind; hop runs carry their
    // channel's distance and boundary period
    int run_kind[kRuns];
    int run_dist[kRuns];
    int run_mod[kRuns];
};

// FROM_LOWER: the images of block p - dist under the +dist hop; FROM_UPPER: of block p + dist
// under the -dist hop; UP / DOWN: one phonon more / less at the exciton site; EMPTY: no run.
enum RunKind : int { RK_SELF = 0, RK_FROM_LOWER = 1, RK_FROM_UPPER = 2, RK_UP = 3, RK_DOWN = 4, RK_EMPTY = 5 };

// The standard runs: self, channel 0 from below and above, phonon up and down (the whole
// Hamiltonian of the chain).
inline void merge_spec_standard(MergeWs& w, const ModelDev& m) {
    const int kinds[kRuns] = {RK_SELF, RK_FROM_LOWER, RK_FROM_UPPER, RK_UP, RK_DOWN};
    for (int j = 0; j < kRuns; ++j) {
        w.run_kind[j] = kinds[j];
        w.run_dist[j] = m.hop_dist[0];
        w.run_mod[j] = m.hop_mod[0];
    }
}

// Self run plus the hop channels ca and cb (cb < 0: none) from below and above.
inline void merge_spec_hops(MergeWs& w, const ModelDev& m, int ca, int cb) {
    w.run_kind[0] = RK_SELF;
    w.run_kind[1] = RK_FROM_LOWER;
    w.run_kind[2] = RK_FROM_UPPER;
    w.run_kind[3] = cb >= 0 ? RK_FROM_LOWER : RK_EMPTY;
    w.run_kind[4] = cb >= 0 ? RK_FROM_UPPER : RK_EMPTY;
    for (int j = 0; j < kRuns; ++j) {
        const int ch = j <= 2 ? ca : (cb >= 0 ? cb : ca);
        w.run_dist[j] = m.hop_dist[ch];
        w.run_mod[j] = m.hop_mod[ch];
    }
}

// Merge passes that cover every channel: the standard pass, then one per two further channels.
inline int merge_passes(const ModelDev& m) { return 1 + (m.nhop - 1 + 1) / 2; }

struct MergeOut {
    uint64_t* keys;
    int* blk;
    int64_t cap;
    // assemble only
    uint32_t* meta;
    int* nbr;        // [4][nbr_cap]
    int64_t nbr_cap;
    // assemble and split expansion: output index of every run element, -1 for holes;
    // [kRuns][map_cap], indexed by the element's source index (in X for the self run, in Y
    // for the image runs)
    int* maps;
    int64_t map_cap;
    // split expansion only: the "new part" -- output states whose group holds no element
    // of the self run -- as a sorted, blocked basis, and each one's output index
    uint64_t* new_keys;
    int* new_blk;
    int* new_to_out;
    int64_t new_cap;
    // assemble: the neighbour fill that follows writes every row of a self-run state whole,
    // so the assembly initialises only the other rows (their entries arrive one by one)
    int self_rows_filled;
    // assemble (optional, nbr_cap bytes): 1 where the output state has a self-run element
    uint8_t* self_flag;
};

// Merge modes.  EXPAND: keys only.  ASSEMBLE: keys, the H rows' metadata and neighbour
// table (through the maps).  EXPAND_SPLIT: an expansion that also writes the maps and the
// new part, so that the following assembly needs the images of the new part only
// (the images of the rest are already in this expansion's output).
enum MergeMode : int { MERGE_EXPAND = 0, MERGE_ASSEMBLE = 1, MERGE_EXPAND_SPLIT = 2 };

// Tiling constants by key width.  merge_stride(nw) is the largest stride (a tile's element
// indices fit 12 bits); any multiple of 16 down to kMinMergeStride works (paces_set_tuning),
// smaller tiles trading splitter work for more resident blocks.  The untuned choices for one
// or two key words, measured on the 2^22 chain: stride 160 for the expansions (three blocks
// per SM), 192 for the assembly.
__host__ __device__ constexpr int merge_stride(int nw) { return nw <= 2 ? 240 : (nw <= 4 ? 128 : 64); }
__host__ __device__ constexpr int merge_default_stride(int nw) { return nw <= 2 ? 160 : (nw <= 4 ? 128 : 64); }
__host__ __device__ constexpr int merge_default_assemble_stride(int nw) { return nw <= 2 ? 192 : (nw <= 4 ? 128 : 64); }
constexpr int kMinMergeStride = 64;
// Splitter intervals per tile: 12 measured faster than 8, 10, 14 and 16 on the 2^22 chain
// (larger tiles spread each thread's merge-path searches over more elements; smaller ones fit
// more blocks per SM).
constexpr int kMergeGroup = 12;
// A tile holds the merged range of kMergeGroup consecutive splitters; every run contributes
// fewer than (its splitters in the range + 1) * stride elements, so at most
// (kMergeGroup + kRuns) * stride elements in total.
__host__ __device__ constexpr int merge_tmax(int stride) { return (kMergeGroup + kRuns) * stride; }

// Splitter capacity for inputs of up to in_cap states at any stride >= kMinMergeStride.
inline int64_t merge_split_cap(int64_t in_cap, int nw, int L) {
    (void)nw;
    return kRuns * (in_cap / kMinMergeStride + 1) + int64_t(kRuns) * L + 8;
}
inline int64_t merge_tile_cap(int64_t split_cap, int L) { return split_cap / kMergeGroup + L + 8; }
// Bytes of one tile descriptor (any key width).
constexpr size_t merge_desc_bytes() { return 320; }

// X feeds the self run, Y (null: X) the four image runs.  ceiling_out (optional) receives the
// number of ceiling holes of the up run, or has it added (ceiling_add).  An assembly with
// Y != X leaves the neighbour table to launch_nbr_fill_split.
int launch_merge(int nw, int mode, int stride, const ModelDev& m, const uint64_t* x_keys, const int* x_blk,
                 const uint64_t* y_keys, const int* y_blk, const MergeWs& ws, const MergeOut& out,
                 int* ceiling_out, int ceiling_add, int* status, int num_sms, cudaStream_t st);

// Neighbour table of a lattice with several hopping channels after the assembly's passes
// (pass_maps[k]: the maps of pass k; see nbr_fill_multi_kernel).  xnbr: [nhop-1][nbr_cap] int2.
int launch_nbr_fill_multi(const ModelDev& m, const int* x_blk, const int* const* pass_maps, int passes, int64_t map_cap,
                          int* nbr, int* xnbr, int64_t nbr_cap, int num_sms, cudaStream_t st);

// Neighbour table after a split expansion (maps_e, new part N with new_to_out) and the
// assembly of its output with the images of N (maps_s): every state of the expansion's
// input P and of N is a source.  p_blk / n_blk: block offsets of P and N.  self_flag: the
// assembly's MergeOut::self_flag (rows of the expansion's output, which carry their reverse
// entries themselves).
int launch_nbr_fill_split(const ModelDev& m, const int* p_blk, const int* n_blk, const int* maps_e,
                          const int* maps_s, const int* new_to_out, const uint8_t* self_flag, int64_t map_cap,
                          int* nbr, int64_t nbr_cap, int num_sms, cudaStream_t st);

}  // namespace paces
