// Exact partition-search transposition table, one per solver lane.
//
// Layout (per lane: 2^tt_log2 buckets of 320 bytes, 64-byte aligned):
//   tag[16]   one 64-byte line, read by a probe as four 128-bit loads
//   e[16]     16-byte entries (w0, w1)
// A tag is hash bits 48..63 (16) | tricks left (4) | way of its entry (4) | generation (6) |
// leader (2), 0 = empty; tags stay in age order (newest first) while entries stay in
// place, so a store rewrites one tag line and one entry. The entry packing
//   w0: q = hash bits 9..47 (39) | lb (4) | ub (4) | best card (6, 63 none) | owners 48..57
//   w1: relevant-card counts per suit (4 bits each) | owners 0..47
// and the eviction rule (least 2*left + age, other generations first) are the
// reference's (src/dd.h:87-111, 325-350, 438-532): both decide which positions the TT
// answers and so the node counts, which the tests compare one for one.
#pragma once
#include "ddg_bits.cuh"

namespace ddg {

enum { TT_WAYS = 16, GEN_BITS = 6, Q_BITS = 39, MAX_REL = 29, TT_MIN_LOG2 = 9 };

#ifndef DDG_TT_SIG
struct alignas(64) TTBucket {
  u32 tag[TT_WAYS];
  u64 e[TT_WAYS][2];
};
static_assert(sizeof(TTBucket) == 320, "bucket is 5 x 64 bytes");
#else
// Signature entries (-DDDG_TT_SIG, libddg_sig.so; the reference's -DDD_TT_SIG build,
// src/dd.h:74-85,352-437): an entry keeps a 64-bit hash of its key (owner patterns of the
// relevant cards, suit lengths, tag) instead of the key, in 12 bytes:
//   sig (two words) | meta = relevant-card counts (4 bits per suit) | lb (4) | ub (4) | best card (6)
// A bucket is then four 64-byte lines, and any number of relevant cards can be stored. It
// is not strictly exact: a wrong hit needs two keys with the same tag and the same hash.
struct alignas(64) TTBucket {
  u32 tag[TT_WAYS];
  u32 e[TT_WAYS][3];
};
static_assert(sizeof(TTBucket) == 256, "bucket is 4 x 64 bytes");
#endif

// Trick-start key of a position: what the TT needs to look it up and to store it.
struct NodeKey {
  u64 code[4];  // suit_codes()
  u64 all;      // cards in play
  u64 lens;     // length_key()
  u64 q;        // hash bits 9..47
  u32 bucket;   // hash bits 0..tt_log2-1
  u32 tag;      // tag without its way
};

DDG_CALL NodeKey make_key(Hands hs, int leader, int left, u32 gen, u32 mask) {
  const u64* h = hs.h;
  NodeKey k;
  suit_codes(h, k.code);
  k.all = all_cards(h);
  k.lens = length_key(h);
  u64 x = key_hash(k.lens, leader);
  k.bucket = (u32)x & mask;
  k.q = (x >> 9) & ((1ull << Q_BITS) - 1);
  k.tag = ((u32)(x >> 32) & 0xFFFF0000u) | ((u32)left << 12) | (gen << 2) | (u32)leader;
  return k;
}

struct ProbeOut {  // a probe's answer (1, 0, or -1 = unknown), best-move hint, relevant cards
  int hit, hint;
  u64 rel;
};

// Traffic counters of the TT (bytes = what the roofline counts as algorithmic bytes).
// Kept per launch per lane, in shared memory on the GPU.
struct TTStats {
  u64 bytes;  // tag lines and entries read + written
  u32 probes, hits, stores;
  u32 entry_reads;  // tag-matched entries a probe read (16 bytes each)
};

DDG_HD void tags_load(const TTBucket* b, u32* t) {
#ifdef __CUDA_ARCH__
  const uint4* v = reinterpret_cast<const uint4*>(b->tag);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint4 x = v[k];
    t[4 * k] = x.x;
    t[4 * k + 1] = x.y;
    t[4 * k + 2] = x.z;
    t[4 * k + 3] = x.w;
  }
#else
  for (int k = 0; k < TT_WAYS; k++) t[k] = b->tag[k];
#endif
}
DDG_HD void tags_store(TTBucket* b, const u32* t) {
#ifdef __CUDA_ARCH__
  uint4* v = reinterpret_cast<uint4*>(b->tag);
#pragma unroll
  for (int k = 0; k < 4; k++) v[k] = make_uint4(t[4 * k], t[4 * k + 1], t[4 * k + 2], t[4 * k + 3]);
#else
  for (int k = 0; k < TT_WAYS; k++) b->tag[k] = t[k];
#endif
}
// Positions (bit k) whose tag equals `tag` apart from the way, and the ways of all 16
// tags packed 4 bits each.
DDG_HD u32 tag_matches(const u32* t, u32 tag, u64& ways) {
  u32 m = 0;
  ways = 0;
#pragma unroll
  for (int k = 0; k < TT_WAYS; k++) {
    m |= (u32)((t[k] & ~0xF00u) == tag) << k;
    ways |= (u64)((t[k] >> 8) & 15) << (4 * k);
  }
  return m;
}

// The way a new entry takes (src/dd.h:330-350): an empty one while the line is not full,
// else the tag of least 2 * tricks left + age, other generations first; that tag leaves
// the line, the tags in front of it move back one and the new tag goes in front. Updates
// the tag line `t` (the caller stores it) and returns the way.
DDG_HD int take_way(u32* t, u64 ways, u32 gen, u32 tag) {
  int pos = TT_WAYS - 1, way;
  if (t[TT_WAYS - 1] != 0) {
    int least = 99;
#pragma unroll
    for (int p = TT_WAYS - 1; p >= 0; p--) {
      int v = ((t[p] >> 2) & 63) != gen ? -1 : 2 * (int)((t[p] >> 12) & 15) + TT_WAYS - 1 - p;
      if (v < least) {
        least = v;
        pos = p;
      }
    }
    way = (int)((ways >> (4 * pos)) & 15);
  } else {
    u32 empty = 0;  // while the line is not full its used tags are positions 0..n-1
#pragma unroll
    for (int p = 0; p < TT_WAYS; p++) empty |= (u32)(t[p] == 0) << p;
    way = low_bit32(empty);
  }
#pragma unroll
  for (int i = TT_WAYS - 1; i > 0; i--)
    if (i <= pos) t[i] = t[i - 1];
  t[0] = tag | ((u32)way << 8);
  return way;
}

#ifndef DDG_TT_SIG
// An entry's first word is stored sealed with its second: e0 = w0 ^ seal(w1). A reader
// unseals with the w1 it read, so a torn entry (words of two different stores, which
// lanes sharing one TT can produce) decodes to a garbled q and fails the probe's key
// check instead of pairing one position's bounds with another's pattern. An untorn entry
// decodes exactly, so every decision, and every node count, is unchanged.
DDG_HD u64 seal(u64 w1) {
  u64 x = (w1 ^ (w1 >> 29)) * 0xBF58476D1CE4E5B9ull;
  return x ^ (x >> 32);
}
DDG_HD void entry_load(const TTBucket* b, int way, u64& w0, u64& w1) {
#ifdef __CUDA_ARCH__
  ulonglong2 x = *reinterpret_cast<const ulonglong2*>(b->e[way]);
  w1 = x.y;
  w0 = x.x ^ seal(x.y);
#else
  w1 = b->e[way][1];
  w0 = b->e[way][0] ^ seal(w1);
#endif
}
DDG_HD void entry_store(TTBucket* b, int way, u64 w0, u64 w1) {
#ifdef __CUDA_ARCH__
  *reinterpret_cast<ulonglong2*>(b->e[way]) = make_ulonglong2(w0 ^ seal(w1), w1);
#else
  b->e[way][0] = w0 ^ seal(w1);
  b->e[way][1] = w1;
#endif
}

// Looks up bounds of the NS tricks still to win. Returns 1 (NS reach `need`), 0 (they do
// not), or -1 (unknown; `hint` = the stored best move of a matching entry, if any).
DDG_CALL ProbeOut tt_probe(const TTBucket* tt, const NodeKey& k, int need, TTStats& st) {
  ProbeOut o;
  o.hit = -1;
  o.hint = -1;
  o.rel = 0;
  const TTBucket* b = tt + k.bucket;
  u32 t[TT_WAYS];
  tags_load(b, t);
  u64 ways;
  u32 m = tag_matches(t, k.tag, ways);
  st.probes++;
  st.bytes += 64;
  int lens_s[4];
#pragma unroll
  for (int s = 0; s < 4; s++) lens_s[s] = code_len(k.code[s]);
  while (m) {
    int pos = low_bit32(m);
    m &= m - 1;
    u64 w0, w1;
    entry_load(b, (int)((ways >> (4 * pos)) & 15), w0, w1);
    st.bytes += 16;
    st.entry_reads++;
    if ((w0 & ((1ull << Q_BITS) - 1)) != k.q) continue;
    u64 owners = (w1 >> 16) | ((w0 >> 53) << 48);
    int off = 0;
    bool same = true;
    int cnt[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      int n = (int)((w1 >> (4 * s)) & 15);
      cnt[s] = n;
      if (n > lens_s[s]) {
        same = false;
      } else {
        u64 stored = ((owners >> off) & ((1ull << (2 * n)) - 1)) | (1ull << (2 * n));
        same = same && (k.code[s] >> (2 * (lens_s[s] - n))) == stored;
      }
      off += 2 * n;
    }
    if (!same) continue;
    int lb = (int)((w0 >> Q_BITS) & 15), ub = (int)((w0 >> (Q_BITS + 4)) & 15);
    if (lb >= need || ub < need) {
      u64 r = 0;
#pragma unroll
      for (int s = 0; s < 4; s++) r |= top_n_cards(k.all, s, cnt[s]);
      o.rel = r;
      st.hits++;
      o.hit = lb >= need ? 1 : 0;
      return o;
    }
    int bm = (int)((w0 >> (Q_BITS + 8)) & 63);
    if (bm != 63) o.hint = bm;
  }
  return o;
}

// Owner patterns of the relevant cards for w1 and w0's top bits; false when more than
// MAX_REL cards are relevant (such results are not stored).
DDG_HD bool pack_owners(const NodeKey& k, u64 rel, u64& w1, u64& hi) {
  u64 counts = 0, owners = 0;
  int total = 0;
#pragma unroll
  for (int s = 0; s < 4; s++) {
    u64 p = rel_pattern(k.code[s], k.all, rel, s);
    int n = code_len(p);
    if (total + n > MAX_REL) return false;
    counts |= (u64)n << (4 * s);
    owners |= (p ^ (1ull << (2 * n))) << (2 * total);
    total += n;
  }
  w1 = counts | (owners << 16);
  hi = (owners >> 48) << 53;
  return true;
}

DDG_HD u64 pack_w0(const NodeKey& k, int lb, int ub, int best, u64 hi) {
  return k.q | (u64)lb << Q_BITS | (u64)ub << (Q_BITS + 4) | (u64)(best < 0 ? 63 : best) << (Q_BITS + 8) | hi;
}

// Stores bounds [lb, ub] of the NS tricks still to win for the class of positions that
// share `rel`'s relevant cards with this one. An entry with the same key is narrowed in
// place; otherwise a way is taken (empty, else other generation, else least
// 2 * tricks left + age) and its tag put in front.
DDG_CALL void tt_store(TTBucket* tt, const NodeKey& k, u32 gen, u64 rel, int lb, int ub, int best,
                       TTStats& st) {
  u64 w1, hi;
  if (!pack_owners(k, rel, w1, hi)) return;
  TTBucket* b = tt + k.bucket;
  u32 t[TT_WAYS];
  tags_load(b, t);
  st.bytes += 64;
  st.stores++;
  u64 ways;
  u32 m = tag_matches(t, k.tag, ways);
  while (m) {
    int pos = low_bit32(m);
    m &= m - 1;
    int way = (int)((ways >> (4 * pos)) & 15);
    u64 e0, e1;
    entry_load(b, way, e0, e1);
    st.bytes += 16;
    if ((e0 & ((1ull << Q_BITS) - 1)) == k.q && e1 == w1 && (e0 >> 53 << 53) == hi) {
      int olb = (int)((e0 >> Q_BITS) & 15), oub = (int)((e0 >> (Q_BITS + 4)) & 15);
      int obest = (int)((e0 >> (Q_BITS + 8)) & 63);
      if (olb > lb) lb = olb;
      if (oub < ub) ub = oub;
      if (best < 0 && obest != 63) best = obest;
#ifdef __CUDA_ARCH__
      reinterpret_cast<u64*>(b->e[way])[0] = pack_w0(k, lb, ub, best, hi) ^ seal(e1);
#else
      b->e[way][0] = pack_w0(k, lb, ub, best, hi) ^ seal(e1);
#endif
      st.bytes += 8;
      return;
    }
  }
  const int way = take_way(t, ways, gen, k.tag);
  tags_store(b, t);
  entry_store(b, way, pack_w0(k, lb, ub, best, hi), w1);
  st.bytes += 64 + 16;
}
#else  // DDG_TT_SIG

DDG_HD u64 sig_mix(u64 x) {  // the splitmix64 finaliser
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Signature of a key: the four owner patterns (each with its leading 1 bit) folded in two
// halves, then the suit lengths, then the tag (src/dd.h:362-367).
DDG_HD u64 key_sig(const NodeKey& k, const u64* p) {
  u64 h = sig_mix((p[0] | p[1] << 27) + 0x9E3779B97F4A7C15ull);
  h = sig_mix(h ^ (p[2] | p[3] << 27));
  return sig_mix(h ^ k.lens) ^ k.tag;
}
DDG_HD void sig_entry_load(const TTBucket* b, int way, u64& sig, u32& meta) {
  sig = (u64)b->e[way][0] | (u64)b->e[way][1] << 32;
  meta = b->e[way][2];
}

DDG_CALL ProbeOut tt_probe(const TTBucket* tt, const NodeKey& k, int need, TTStats& st) {
  ProbeOut o;
  o.hit = -1;
  o.hint = -1;
  o.rel = 0;
  const TTBucket* b = tt + k.bucket;
  u32 t[TT_WAYS];
  tags_load(b, t);
  u64 ways;
  u32 m = tag_matches(t, k.tag, ways);
  st.probes++;
  st.bytes += 64;
  int lens_s[4];
#pragma unroll
  for (int s = 0; s < 4; s++) lens_s[s] = code_len(k.code[s]);
  while (m) {
    int pos = low_bit32(m);
    m &= m - 1;
    u64 sig;
    u32 meta;
    sig_entry_load(b, (int)((ways >> (4 * pos)) & 15), sig, meta);
    st.bytes += 12;
    st.entry_reads++;
    u64 p[4];
    int cnt[4];
    bool fit = true;
#pragma unroll
    for (int s = 0; s < 4; s++) {
      cnt[s] = (int)(meta >> (4 * s)) & 15;
      fit = fit && cnt[s] <= lens_s[s];
      p[s] = fit ? k.code[s] >> (2 * (lens_s[s] - cnt[s])) : 0;
    }
    if (!fit || key_sig(k, p) != sig) continue;
    int lb = (int)(meta >> 16) & 15, ub = (int)(meta >> 20) & 15;
    if (lb >= need || ub < need) {
      u64 r = 0;
#pragma unroll
      for (int s = 0; s < 4; s++) r |= top_n_cards(k.all, s, cnt[s]);
      o.rel = r;
      st.hits++;
      o.hit = lb >= need ? 1 : 0;
      return o;
    }
    int bm = (int)(meta >> 24) & 63;
    if (bm != 63) o.hint = bm;
  }
  return o;
}

// Stores bounds under the signature of the relevant cards' owner patterns (no limit on
// their number): an entry with the same signature and counts is narrowed, else a way is
// taken as in the exact table.
DDG_CALL void tt_store(TTBucket* tt, const NodeKey& k, u32 gen, u64 rel, int lb, int ub, int best,
                       TTStats& st) {
  u64 p[4];
  u32 counts = 0;
#pragma unroll
  for (int s = 0; s < 4; s++) {
    p[s] = rel_pattern(k.code[s], k.all, rel, s);
    counts |= (u32)code_len(p[s]) << (4 * s);
  }
  const u64 sig = key_sig(k, p);
  TTBucket* b = tt + k.bucket;
  u32 t[TT_WAYS];
  tags_load(b, t);
  st.bytes += 64;
  st.stores++;
  u64 ways;
  u32 m = tag_matches(t, k.tag, ways);
  int way = -1;
  while (m && way < 0) {
    int pos = low_bit32(m);
    m &= m - 1;
    const int w = (int)((ways >> (4 * pos)) & 15);
    u64 osig;
    u32 ometa;
    sig_entry_load(b, w, osig, ometa);
    st.bytes += 12;
    if (osig == sig && (ometa & 0xFFFFu) == counts) {
      const int olb = (int)(ometa >> 16) & 15, oub = (int)(ometa >> 20) & 15, obest = (int)(ometa >> 24) & 63;
      if (olb > lb) lb = olb;
      if (oub < ub) ub = oub;
      if (best < 0 && obest != 63) best = obest;
      way = w;
    }
  }
  if (way < 0) {
    way = take_way(t, ways, gen, k.tag);
    tags_store(b, t);
    b->e[way][0] = (u32)sig;
    b->e[way][1] = (u32)(sig >> 32);
    st.bytes += 64 + 8;
  }
  b->e[way][2] = counts | (u32)lb << 16 | (u32)ub << 20 | (u32)(best < 0 ? 63 : best) << 24;
  st.bytes += 4;
}
#endif  // DDG_TT_SIG

// Next generation of a lane's TT; at the wrap all tags are cleared.
DDG_CALL u32 tt_next_gen(TTBucket* tt, u32 mask, u32 gen) {
  gen++;
  if (gen >= (1u << GEN_BITS)) {
    u32 zero[TT_WAYS];
#pragma unroll
    for (int k = 0; k < TT_WAYS; k++) zero[k] = 0;
    for (u32 i = 0; i <= mask; i++) tags_store(tt + i, zero);
    gen = 1;
  }
  return gen;
}

}  // namespace ddg
