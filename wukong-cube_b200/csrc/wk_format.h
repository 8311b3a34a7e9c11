// GStore format shared by the host builder, the C-ABI layer and the device kernels.
//
// The key/value layout is Wukong's static segment store, kept bit-for-bit so that a store
// exported by the reference engine can be uploaded unchanged:
//   * a slot (vertex_t, src/core/store/vertex.hpp:176-179) is 16 bytes: a 64-bit key word and
//     a 64-bit pointer word;
//   * key word = ikey_t{dir:1, pid:17, vid:46} (vertex.hpp:66-69).  With GCC's little-endian
//     bitfield allocation that is (vid << 18) | (pid << 1) | dir, which is also exactly the
//     integer ikey_t::hash() feeds to the mixer (vertex.hpp:106-116);
//   * pointer word = iptr_t{size:28, off:34, type:2} (vertex.hpp:133-140), i.e.
//     size in bits 0..27, off in bits 28..61, type in bits 62..63;
//   * buckets hold ASSOCIATIVITY = 8 slots (kvstore.hpp:83); slots 0..6 hold keys, slot 7 is
//     the chain link whose key.vid is the absolute id of the next bucket (kvstore.hpp:182-196,
//     292-314); an all-zero key word is an empty slot (vertex.hpp:96);
//   * a segment is one (pid, dir) pair for normal keys, or the index segment of one direction
//     for keys with vid == 0 (segment_meta.hpp:168-178); its bucket is
//     bucket_start + hash(key) % num_buckets (kvstore.hpp:260-268);
//   * an edge (edge_t, vertex.hpp:182) is one 32-bit vertex/type id.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define WK_HD __host__ __device__ __forceinline__
#else
#define WK_HD inline
#endif

namespace wk {

constexpr int kAssoc = 8;              // slots per bucket
constexpr int kNbitsDir = 1;
constexpr int kNbitsIdx = 17;          // predicate / type id width
constexpr int kNbitsVid = 46;
constexpr int kNbitsSize = 28;
constexpr int kNbitsOff = 34;
constexpr uint32_t kPredicateId = 0;   // vertex.hpp:52-53
constexpr uint32_t kTypeId = 1;
constexpr uint32_t kBlankId = 0xFFFFFFFFu;   // type.hpp:41 (32-bit sid_t)
constexpr uint32_t kVidMin = 1u << kNbitsIdx;
constexpr int kIn = 0;                 // type.hpp:50, enum dir_t { IN = 0, OUT }
constexpr int kOut = 1;

WK_HD bool is_tpid(int64_t id) { return id > 1 && id < (1 << kNbitsIdx); }   // vertex.hpp:55
WK_HD bool is_vid(int64_t id) { return id >= (1 << kNbitsIdx); }             // vertex.hpp:57

WK_HD uint64_t make_key(uint64_t vid, uint64_t pid, uint64_t dir) {
    return (vid << (kNbitsIdx + kNbitsDir)) | (pid << kNbitsDir) | dir;
}
WK_HD uint64_t key_vid(uint64_t k) { return k >> (kNbitsIdx + kNbitsDir); }
WK_HD uint32_t key_pid(uint64_t k) { return (uint32_t)((k >> kNbitsDir) & ((1u << kNbitsIdx) - 1)); }
WK_HD uint32_t key_dir(uint64_t k) { return (uint32_t)(k & 1u); }

WK_HD uint64_t make_ptr(uint64_t size, uint64_t off) { return size | (off << kNbitsSize); }
WK_HD uint64_t ptr_size(uint64_t p) { return p & ((1ull << kNbitsSize) - 1); }
WK_HD uint64_t ptr_off(uint64_t p) { return (p >> kNbitsSize) & ((1ull << kNbitsOff) - 1); }

// Thomas Wang's 64-bit integer mix, the hash Wukong uses for bucket placement
// (src/utils/math.hpp:59-68, device copy src/gpu/gpu_hash.cu:36-54).  It must be the same
// function for a store built by either side to be probed by the other.
WK_HD uint64_t hash_u64(uint64_t key) {
    key = (~key) + (key << 21);
    key = key ^ (key >> 24);
    key = (key + (key << 3)) + (key << 8);
    key = key ^ (key >> 14);
    key = (key + (key << 2)) + (key << 4);
    key = key ^ (key >> 28);
    key = key + (key << 31);
    return key;
}

// One slot of the key table (vertex_t).
struct alignas(16) Slot {
    uint64_t key;
    uint64_t ptr;
};
static_assert(sizeof(Slot) == 16, "slot must be 16 bytes");

// Where one segment lives inside the uploaded slot and edge arrays.  Only the fields the
// probe needs; the rest of rdf_seg_meta_t (segment_meta.hpp:87-154) is bookkeeping.
struct SegDesc {
    uint64_t bucket_start;   // absolute bucket id of the segment's main-header region
    uint64_t num_buckets;    // hash space of the segment (0 = segment absent / empty)
    uint64_t magic;          // floor((2^64 - 1) / num_buckets): Barrett reciprocal of the modulo
    uint64_t num_edges;      // number of edges of the segment (informational)
};

WK_HD uint64_t barrett_magic(uint64_t nb) { return nb ? ~0ull / nb : 0; }

// hash % nb without a 64-bit division (Barrett, "Implementing the Rivest Shamir and Adleman
// public key encryption algorithm on a standard digital signal processor", CRYPTO 1986):
// with m = floor((2^64 - 1) / nb) the estimate q = floor(h * m / 2^64) is at most one short of
// floor(h / nb), so one conditional subtraction gives the exact remainder.
WK_HD uint64_t mod_barrett(uint64_t h, uint64_t nb, uint64_t m) {
#if defined(__CUDA_ARCH__)
    uint64_t q = __umul64hi(h, m);
#else
    uint64_t q = (uint64_t)(((unsigned __int128)h * m) >> 64);
#endif
    uint64_t r = h - q * nb;
    if (r >= nb) r -= nb;
    if (r >= nb) r -= nb;
    return r;
}

}  // namespace wk
