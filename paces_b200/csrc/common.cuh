// Shared device definitions of libpaces_b200: model descriptor, packed Fock keys,
// key comparison, status reporting and bounded waits.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/paces_b200.h"

namespace paces {

constexpr int kMaxSites = PACES_MAX_SITES;
constexpr int kMaxKeyWords = 8;
constexpr int kRuns = 5;  // candidate runs per exciton block: self, from-left, from-right, up, down
constexpr int kMaxHop = 6;  // hopping channels: up to 3 lattice dimensions x 2 hopping terms
enum Run : int { RUN_SELF = 0, RUN_FROM_LEFT = 1, RUN_FROM_RIGHT = 2, RUN_UP = 3, RUN_DOWN = 4 };
// neighbour slots of the H table (paces_hmat.nbr)
enum Slot : int { NB_LEFT = 0, NB_RIGHT = 1, NB_DOWN = 2, NB_UP = 3 };

// Model constants passed by value to every kernel (fits the 32 KB parameter space).
struct ModelDev {
    int L;             // sites == exciton positions
    int nw;            // uint64 words per key
    int periodic;
    int has_site_eps;
    double eps_sys, hbar_omega, delta_eps, J, g;
    uint8_t word[kMaxSites];   // word holding site s
    uint8_t shift[kMaxSites];  // bit position of the field's least significant bit
    uint8_t bits[kMaxSites];   // field width
    uint16_t maxd[kMaxSites];  // max_ho_dims[s]
    double site_eps[kMaxSites];
    // plane[q][b]: the bits of word q that are bit b of some field (b < max_bits), so the
    // total phonon count of a key is sum_{q,b} popc(w[q] & plane[q][b]) << b
    int max_bits;
    uint64_t plane[kMaxKeyWords][8];
    // Hopping channels.  Channel 0 is the nearest-neighbour hop along the first lattice
    // dimension (the chain's only channel); channels 1.. are the further lattice dimensions
    // of the "hopping" term and then the dimensions of the "hopping2" term.  A channel moves
    // the exciton by +-hop_dist; with open boundaries the +dist hop from p exists when
    // p % hop_mod < hop_mod - hop_dist (p stays in its row of the lattice).
    int nhop;
    int hop_dist[kMaxHop];
    int hop_mod[kMaxHop];
    int hop_term[kMaxHop];      // 0: hopping (J), 1: hopping2 (J2)
    double J2;
    // per term, the row's hopping elements in increasing column (= position) order:
    // channel << 1 | side, side 0 = the neighbour at p - dist, 1 = at p + dist
    int hop_n[2];
    int8_t hop_ord[2][2 * kMaxHop];
    // extra channels' neighbour table of the H a kernel reads ([nhop-1][xcap] int2: lower,
    // upper neighbour), set per launch; null when nhop == 1
    const int2* xnbr;
    int64_t xcap;
};

// Blocks for a grid-stride pass over at most `items` elements handled `per_block` at a time:
// a full wave (`max_blocks`) for large problems, fewer for small ones (the trajectories of a
// batch), so that a small launch does not pay for a wave of idle blocks.
inline int grid_for(int64_t items, int per_block, int max_blocks) {
    const int64_t b = (items + per_block - 1) / per_block;
    return int(b < 1 ? 1 : (b > max_blocks ? max_blocks : b));
}

// Whether the exciton at p has a neighbour through channel ch on side `up` (1: +dist, 0: -dist).
__host__ __device__ __forceinline__ bool hop_exists(const ModelDev& m, int ch, int p, int up) {
    if (m.periodic) return true;
    const int d = m.hop_dist[ch], md = m.hop_mod[ch];
    return up ? (p % md < md - d) : (p % md >= d);
}

template <int NW>
struct Key {
    uint64_t w[NW];
};

template <int NW>
__device__ __forceinline__ Key<NW> load_key(const uint64_t* __restrict__ base, int64_t i) {
    Key<NW> k;
    const uint64_t* q = base + i * NW;
    if constexpr (NW % 2 == 0) {
#pragma unroll
        for (int w = 0; w < NW; w += 2) {
            ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(q + w));
            k.w[w] = v.x;
            k.w[w + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int w = 0; w < NW; ++w) k.w[w] = __ldg(q + w);
    }
    return k;
}

template <int NW>
__device__ __forceinline__ void store_key(uint64_t* __restrict__ base, int64_t i, const Key<NW>& k) {
    uint64_t* q = base + i * NW;
    if constexpr (NW % 2 == 0) {
#pragma unroll
        for (int w = 0; w < NW; w += 2)
            *reinterpret_cast<ulonglong2*>(q + w) = make_ulonglong2(k.w[w], k.w[w + 1]);
    } else {
#pragma unroll
        for (int w = 0; w < NW; ++w) q[w] = k.w[w];
    }
}

// -1 / 0 / +1 lexicographic comparison of the word sequences.
template <int NW>
__device__ __forceinline__ int key_cmp(const Key<NW>& a, const Key<NW>& b) {
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        if (a.w[w] != b.w[w]) return a.w[w] < b.w[w] ? -1 : 1;
    }
    return 0;
}

template <int NW>
__device__ __forceinline__ bool key_eq(const Key<NW>& a, const Key<NW>& b) {
    bool eq = true;
#pragma unroll
    for (int w = 0; w < NW; ++w) eq &= (a.w[w] == b.w[w]);
    return eq;
}

template <int NW>
__device__ __forceinline__ uint32_t get_field(const ModelDev& m, const Key<NW>& k, int s) {
    const uint64_t mask = (uint64_t(1) << m.bits[s]) - 1;
    // a mask per word instead of a select: the compiler would turn a select on the word index
    // into an indexed access of a local copy of the key
    const int ws = m.word[s];
    uint64_t word = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) word |= k.w[w] & (uint64_t(0) - uint64_t(w == ws));
    return uint32_t((word >> m.shift[s]) & mask);
}

// field s += delta (caller guarantees no overflow out of the field)
template <int NW>
__device__ __forceinline__ void add_field(const ModelDev& m, Key<NW>& k, int s, int delta) {
    const uint64_t one = uint64_t(1) << m.shift[s];
    const uint64_t d = delta > 0 ? one : (uint64_t(0) - one);
    const int ws = m.word[s];
#pragma unroll
    for (int w = 0; w < NW; ++w) k.w[w] += d & (uint64_t(0) - uint64_t(w == ws));
}

// Sum of all occupation fields: one popcount per word and bit plane.
template <int NW>
__device__ __forceinline__ uint32_t total_phonons(const ModelDev& m, const Key<NW>& k) {
    uint32_t t = 0;
#pragma unroll
    for (int q = 0; q < NW; ++q) {
#pragma unroll 8
        for (int b = 0; b < m.max_bits; ++b) t += uint32_t(__popcll(k.w[q] & m.plane[q][b])) << b;
    }
    return t;
}

// ---- status words ------------------------------------------------------------------------
__device__ __forceinline__ void raise_status(int* status, int code) {
    if (status) atomicCAS(status, 0, code);
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Upper bound on any device-side wait (look-back, grid barrier): 2 s.
constexpr uint64_t kWaitLimitNs = 2000000000ull;

// Block id of `i` in block offsets blk[0..L] (blk sorted): largest p with blk[p] <= i.
__device__ __forceinline__ int block_of(const int* blk, int L, int64_t i) {
    int lo = 0, hi = L - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (blk[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

}  // namespace paces
