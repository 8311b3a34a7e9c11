// Internal declarations shared by the host-side translation units of libwukong_b200.
#pragma once
#include <stdint.h>

#include <vector>

#include "../../include/wukong_b200.h"
#include "wk_format.h"

namespace wk {

int synth_generate(const wk_synth_params& p, std::vector<uint32_t>& out, wk_synth_vocab& v);

// Probe a host copy of the key table (the same walk the device kernels do).
// Returns the pointer word of the key, or 0 when the key is absent.
inline uint64_t host_probe(const Slot* slots, uint64_t n_buckets_total, const SegDesc& seg,
                           uint64_t key, int* corrupt) {
    if (seg.num_buckets == 0) return 0;
    uint64_t b = seg.bucket_start + mod_barrett(hash_u64(key), seg.num_buckets, seg.magic);
    for (uint64_t hop = 0; hop <= n_buckets_total; ++hop) {
        if (b >= n_buckets_total) {
            if (corrupt) *corrupt = 1;
            return 0;
        }
        const Slot* bk = slots + b * kAssoc;
        for (int i = 0; i < kAssoc - 1; ++i)
            if (bk[i].key == key) return bk[i].ptr;
        if (bk[kAssoc - 1].key == 0) return 0;
        b = key_vid(bk[kAssoc - 1].key);
    }
    if (corrupt) *corrupt = 1;
    return 0;
}

// Map from segid_t to the segment list, for host lookups and plan resolution.
struct SegIndex {
    std::vector<int32_t> normal;   // [pid * 2 + dir] -> segment number, -1 if none
    int32_t index_seg[2] = {-1, -1};
    void build(const wk_seg_meta* segs, uint32_t n);
    // Segment of a key: vid == 0 -> index segment (segment_meta.hpp:168-178).
    int32_t find(uint64_t vid, uint32_t pid, int dir) const {
        if (dir < 0 || dir > 1) return -1;
        if (vid == 0) return index_seg[dir];
        if (pid >= (1u << kNbitsIdx)) return -1;
        return normal[(size_t)pid * 2 + dir];
    }
};

inline SegDesc to_desc(const wk_seg_meta& m) {
    SegDesc d;
    d.bucket_start = m.bucket_start;
    d.num_buckets = m.num_buckets;
    d.magic = barrett_magic(m.num_buckets);
    d.num_edges = m.num_edges;
    return d;
}

}  // namespace wk

// Host-built static store (opaque in the C ABI).
struct wk_gstore {
    std::vector<wk::Slot> slots;
    std::vector<uint32_t> edges;
    std::vector<wk_seg_meta> segs;
    wk::SegIndex index;
    uint64_t n_keys = 0;
};
