// Card model, bit primitives and the transposition-table key of a position.
//
// Cards are bit (suit * 16 + rank) of a uint64: suit 0..3 = S,H,D,C, rank 0..12 = 2..A.
// Seats 0..3 = N,E,S,W (NS = even seats). Strains 0..4 = C,D,H,S,NT; the trump suit of
// strain k is 3 - k, and -1 for NT. This is the reference's card model
// (src/dd.h:13-14, 893), kept so its 32-byte hand-mask records are read unchanged.
//
// Everything here compiles for the host (g++) and for sm_100a (nvcc): the host build is
// only used by the tests to replay the stage machine on the CPU.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define DDG_HD __host__ __device__ __forceinline__
// Heavy routines stay out of line on the GPU: one copy each keeps the kernel's code small
// enough for the instruction caches, which lanes in different stages otherwise thrash.
#define DDG_CALL __host__ __device__ __noinline__
#else
#define DDG_HD static inline
#define DDG_CALL static
#endif

namespace ddg {

typedef uint64_t u64;
typedef uint32_t u32;

DDG_HD int popc(u64 x) {
#ifdef __CUDA_ARCH__
  return __popcll(x);
#else
  return __builtin_popcountll(x);
#endif
}
DDG_HD int popc32(u32 x) {
#ifdef __CUDA_ARCH__
  return __popc(x);
#else
  return __builtin_popcount(x);
#endif
}
// Highest / lowest set bit; x != 0.
DDG_HD int top_bit(u64 x) {
#ifdef __CUDA_ARCH__
  return 63 - __clzll((long long)x);
#else
  return 63 - __builtin_clzll(x);
#endif
}
DDG_HD int low_bit(u64 x) {
#ifdef __CUDA_ARCH__
  return __ffsll((long long)x) - 1;
#else
  return __builtin_ctzll(x);
#endif
}
DDG_HD int low_bit32(u32 x) {
#ifdef __CUDA_ARCH__
  return __ffs((int)x) - 1;
#else
  return __builtin_ctz(x);
#endif
}

// Asks for a line to be brought into L1 (GPU) ahead of a dependent load; no-op on the host.
DDG_HD void prefetch_l1(const void* p) {
#ifdef __CUDA_ARCH__
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
#else
  (void)p;
#endif
}
DDG_HD void prefetch_l2(const void* p) {
#ifdef __CUDA_ARCH__
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
#else
  (void)p;
#endif
}

DDG_HD u64 card_bit(int c) { return (u64)1 << c; }
DDG_HD u64 suit_cards(int s) { return (u64)0x1FFF << (16 * s); }
DDG_HD int card_suit(int c) { return c >> 4; }
DDG_HD int lho_of(int h) { return (h + 1) & 3; }
DDG_HD int partner_of(int h) { return (h + 2) & 3; }
DDG_HD int rho_of(int h) { return (h + 3) & 3; }
DDG_HD bool ns_side(int h) { return (h & 1) == 0; }
DDG_HD int strain_trump(int strain) { return strain == 4 ? -1 : 3 - strain; }

// The four hands, passed by value to out-of-line routines (eight registers).
struct Hands {
  u64 h[4];
};

// hands[i] for a run-time seat i, written as selects so the four hands stay in registers.
DDG_HD u64 hand_at(const u64* h, int i) {
  u64 a = (i & 1) ? h[1] : h[0];
  u64 b = (i & 1) ? h[3] : h[2];
  return (i & 2) ? b : a;
}
DDG_HD void toggle_card(u64* h, int seat, int card) {
  u64 m = card_bit(card);
  h[0] ^= seat == 0 ? m : 0;
  h[1] ^= seat == 1 ? m : 0;
  h[2] ^= seat == 2 ? m : 0;
  h[3] ^= seat == 3 ? m : 0;
}
DDG_HD u64 all_cards(const u64* h) { return h[0] | h[1] | h[2] | h[3]; }

// Seat holding `card` (0 when no hand holds it), without a search over seats.
DDG_HD int holder_of(const u64* h, int card) {
  return (int)((h[1] >> card) & 1) + 2 * (int)((h[2] >> card) & 1) + 3 * (int)((h[3] >> card) & 1);
}

// Suit lengths, 4 bits per (hand, suit): hand h suit s at bit 60 - 16h - 4s. This layout is
// the hashed key of the TT (src/dd.h:177-189), so it is kept bit for bit.
DDG_HD u64 length_key(const u64* h) {
  u64 k = 0;
#pragma unroll
  for (int p = 0; p < 4; p++) {
    u32 lo = (u32)h[p], hi = (u32)(h[p] >> 32);
    u32 v = (u32)popc32(lo & 0xFFFFu) << 12 | (u32)popc32(lo >> 16) << 8 |
            (u32)popc32(hi & 0xFFFFu) << 4 | (u32)popc32(hi >> 16);
    k |= (u64)v << (48 - 16 * p);
  }
  return k;
}
DDG_HD int len_of(u64 lens, int h, int s) { return (int)((lens >> (60 - 16 * h - 4 * s)) & 15); }

// Hash of (lengths, leader), a bijection of lens ^ leader<<62 (odd multiplies and
// xor-shifts are invertible). Bucket, tag and q are slices of it; the reference's TT
// (src/dd.h:191-196) uses the same function, which keeps node counts identical.
DDG_HD u64 key_hash(u64 lens, int leader) {
  u64 x = (lens ^ ((u64)leader << 62)) * 0x9E3779B97F4A7C15ull;
  x ^= x >> 29;
  x *= 0xBF58476D1CE4E5B9ull;
  return x ^ (x >> 32);
}

// Compress within 16-bit lanes (Hacker's Delight, 2nd ed., section 7-4, "compress" by
// parallel suffix): the bits of d0 and d1 selected by m move down to the low end of their
// lane, keeping their order. Four rounds cover the 16-bit lane width.
DDG_HD void lane_compress(u64& d0, u64& d1, u64 m) {
  const u64 keep1 = 0xFFFEFFFEFFFEFFFEull, keep2 = 0xFFFCFFFCFFFCFFFCull,
            keep4 = 0xFFF0FFF0FFF0FFF0ull, keep8 = 0xFF00FF00FF00FF00ull;
  d0 &= m;
  d1 &= m;
  u64 zeros = (~m << 1) & keep1;  // zeros of m strictly below each bit, counted mod 2 per round
#pragma unroll
  for (int round = 0; round < 4; round++) {
    u64 sfx = zeros ^ ((zeros << 1) & keep1);
    sfx ^= (sfx << 2) & keep2;
    sfx ^= (sfx << 4) & keep4;
    sfx ^= (sfx << 8) & keep8;
    u64 moving = sfx & m;
    int sh = 1 << round;
    m = (m ^ moving) | (moving >> sh);
    u64 t0 = d0 & moving, t1 = d1 & moving;
    d0 = (d0 ^ t0) | (t0 >> sh);
    d1 = (d1 ^ t1) | (t1 >> sh);
    zeros &= ~sfx;
  }
}

// Spreads the low 16 bits of x to the even bit positions (Morton order).
DDG_HD u32 spread_even(u32 x) {
  x &= 0xFFFFu;
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

// Owner code of every suit: the remaining cards of the suit from lowest (bits 0,1) to
// highest, 2 bits each holding the seat, behind a leading 1 bit at 2 * length.
DDG_HD void suit_codes(const u64* h, u64* code) {
  u64 all = all_cards(h);
  u64 b0 = h[1] | h[3], b1 = h[2] | h[3];  // seat bit 0 and bit 1 of every card
  lane_compress(b0, b1, all);
#pragma unroll
  for (int s = 0; s < 4; s++) {
    u32 c0 = (u32)(b0 >> (16 * s)) & 0x1FFFu, c1 = (u32)(b1 >> (16 * s)) & 0x1FFFu;
    int n = popc32((u32)(all >> (16 * s)) & 0x1FFFu);
    code[s] = (u64)(spread_even(c0) | (spread_even(c1) << 1)) | ((u64)1 << (2 * n));
  }
}

DDG_HD int code_len(u64 code) { return top_bit(code) >> 1; }

// The top n remaining cards of suit s (n <= length). Finds the largest r with at least n
// cards at or above rank r by four popcount steps.
DDG_HD u64 top_n_cards(u64 all, int s, int n) {
  u32 a = (u32)(all >> (16 * s)) & 0x1FFFu;
  int r = 0;
#pragma unroll
  for (int step = 8; step; step >>= 1)
    if (popc32(a >> (r + step)) >= n) r += step;
  return (u64)((a >> r) << r) << (16 * s);
}

// Owner pattern (code form) of the cards of suit s at or above its lowest relevant card.
DDG_HD u64 rel_pattern(u64 code, u64 all, u64 rel, int s) {
  u64 r = rel & suit_cards(s);
  if (!r) return 1;
  int low = low_bit(r);
  u64 in = all & suit_cards(s);
  int len = popc(in), above = popc(in >> low);
  return code >> (2 * (len - above));
}

}  // namespace ddg
