/* dd_oracle.c - CPU restatement of the reference's exact double-dummy solve.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA product, never linked into it. Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it
 * (oracle/_build/libddoracle.so).
 *
 * It restates hsperr/dds_gpu's algorithm for the path (src/dd.h, src/dd_bounds.h) in plain
 * C: a recursive null-window search instead of the reference's explicit stack, and plain
 * loops over cards where the reference and the product use bit-parallel tricks (owner
 * codes, suit lengths, run tops, top-n cards). The search order, the bounds, the move
 * weights and the TT rules are the reference's, so both trick tables and search-node
 * counts must equal the reference's. Pinned by: the reference itself compiled here
 * (oracle/_ref, tests/test_oracle.py), the Pgx DDS tables in the reference's
 * data/deals_20k.npy, and an unpruned minimax (ddo_brute) on small endings.
 *
 * Cards: bit suit*16+rank, suits S,H,D,C = 0..3, ranks 2..A = 0..12; seats N,E,S,W;
 * strains C,D,H,S,NT (src/dd.h:13-14). */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef uint32_t u32;

static int popc(u64 x) { return __builtin_popcountll(x); }
static int msb(u64 x) { return 63 - __builtin_clzll(x); }
static int lsb(u64 x) { return __builtin_ctzll(x); }
static u64 bitc(int c) { return (u64)1 << c; }
static u64 suit_mask(int s) { return (u64)0x1FFF << (16 * s); }
static int P_of(int h) { return (h + 2) & 3; }
static int L_of(int h) { return (h + 1) & 3; }
static int R_of(int h) { return (h + 3) & 3; }
static int is_ns(int h) { return (h & 1) == 0; }

/* Seat holding the card, found by asking each hand (src/dd.h:51-53). */
static int owner(const u64* h, int card) {
  for (int p = 0; p < 4; p++)
    if (h[p] >> card & 1) return p;
  return 0;
}

/* ---- TT key (src/dd.h:165-244) ---------------------------------------------------- */

/* 4 bits per (hand, suit) at bit 60 - 16h - 4s (src/dd.h:179-189). */
static u64 lengths(const u64* h) {
  u64 k = 0;
  for (int p = 0; p < 4; p++)
    for (int s = 0; s < 4; s++) k |= (u64)popc(h[p] & suit_mask(s)) << (60 - 16 * p - 4 * s);
  return k;
}

/* src/dd.h:191-196. */
static u64 hash_lens(u64 lens, int leader) {
  u64 x = (lens ^ ((u64)leader << 62)) * 0x9E3779B97F4A7C15ull;
  x ^= x >> 29;
  x *= 0xBF58476D1CE4E5B9ull;
  return x ^ (x >> 32);
}

/* Owners of the remaining cards of each suit, lowest card in bits 0-1, with a leading 1
 * (src/dd.h:162-175), built card by card. */
static void owner_codes(const u64* h, u64* code) {
  for (int s = 0; s < 4; s++) {
    u64 c = 0;
    int j = 0;
    for (int r = 0; r < 13; r++) {
      int card = s * 16 + r;
      for (int p = 0; p < 4; p++)
        if (h[p] >> card & 1) {
          c |= (u64)p << (2 * j);
          j++;
        }
    }
    code[s] = c | (u64)1 << (2 * j);
  }
}

static int code_len(u64 code) { return msb(code) >> 1; }

/* The n highest remaining cards of suit s (src/dd.h:200-205), counted down from the ace. */
static u64 top_cards(u64 all, int s, int n) {
  u64 out = 0;
  for (int r = 12; r >= 0 && n > 0; r--)
    if (all >> (s * 16 + r) & 1) {
      out |= bitc(s * 16 + r);
      n--;
    }
  return out;
}

/* src/dd.h:208-215. */
static u64 pattern(u64 code, u64 all, u64 rel, int s) {
  u64 r = rel & suit_mask(s);
  if (!r) return 1;
  int low = lsb(r), len = 0, n = 0;
  for (int rank = 0; rank < 13; rank++) {
    int card = s * 16 + rank;
    if (all >> card & 1) {
      len++;
      if (card >= low) n++;
    }
  }
  return code >> (2 * (len - n));
}

typedef struct {
  u32 tag[16];
  u64 w0[16], w1[16];
} OBucket;

typedef struct {
  u64 code[4], lens, all, q;
  u32 bucket, tag;
} OKey;

typedef struct {
  u64 hand[4];
  int trump, leader, nplayed, ns_won, left;
  int trick[4];
  OBucket* tt;
  u32 mask, gen;
  u64 nodes;
} OCtx;

#define QBITS 39
#define QMASK ((1ull << QBITS) - 1)

static void make_key(const OCtx* c, OKey* k) {
  owner_codes(c->hand, k->code);
  k->lens = lengths(c->hand);
  k->all = c->hand[0] | c->hand[1] | c->hand[2] | c->hand[3];
  u64 x = hash_lens(k->lens, c->leader);
  k->bucket = (u32)x & c->mask;
  k->q = (x >> 9) & QMASK;
  k->tag = ((u32)(x >> 32) & 0xFFFF0000u) | ((u32)c->left << 12) | (c->gen << 2) | (u32)c->leader;
}

/* src/dd.h:458-493. */
static int tt_probe(const OCtx* c, const OKey* k, int need, u64* rel, int* best) {
  const OBucket* b = c->tt + k->bucket;
  for (int i = 0; i < 16; i++) {
    if ((b->tag[i] & ~0xF00u) != k->tag) continue;
    int way = (b->tag[i] >> 8) & 15;
    u64 w0 = b->w0[way], w1 = b->w1[way];
    if ((w0 & QMASK) != k->q) continue;
    u64 owners = w1 >> 16 | (w0 >> 53) << 48;
    int n[4], off = 0, match = 1;
    for (int s = 0; s < 4; s++) {
      n[s] = (int)(w1 >> (4 * s)) & 15;
      int len = code_len(k->code[s]);
      if (n[s] > len) match = 0;
      else {
        u64 p = (owners >> off & ((1ull << (2 * n[s])) - 1)) | (1ull << (2 * n[s]));
        if ((k->code[s] >> (2 * (len - n[s]))) != p) match = 0;
      }
      off += 2 * n[s];
    }
    if (!match) continue;
    int lb = (int)(w0 >> QBITS) & 15, ub = (int)(w0 >> (QBITS + 4)) & 15;
    if (lb >= need || ub < need) {
      u64 r = 0;
      for (int s = 0; s < 4; s++) r |= top_cards(k->all, s, n[s]);
      *rel = r;
      return lb >= need;
    }
    int bm = (int)(w0 >> (QBITS + 8)) & 63;
    if (bm != 63) *best = bm;
  }
  return -1;
}

/* src/dd.h:330-350: a way for a new tag, which goes in front of the age-ordered line. */
static int tt_slot(const OCtx* c, OBucket* b, u32 tag) {
  int way, pos = 15;
  if (b->tag[15]) {
    int least = 99;
    for (int p = 15; p >= 0; p--) {
      u32 t = b->tag[p];
      int v = ((t >> 2) & 63) != c->gen ? -1 : 2 * (int)((t >> 12) & 15) + 15 - p;
      if (v < least) {
        least = v;
        pos = p;
      }
    }
    way = (b->tag[pos] >> 8) & 15;
  } else {
    way = 0;
    while (b->tag[way]) way++;
  }
  for (int i = pos; i > 0; i--) b->tag[i] = b->tag[i - 1];
  b->tag[0] = tag | ((u32)way << 8);
  return way;
}

/* src/dd.h:441-455, 495-532. */
static void tt_store(OCtx* c, const OKey* k, u64 rel, int lb, int ub, int best) {
  u64 counts = 0, owners = 0;
  int total = 0;
  for (int s = 0; s < 4; s++) {
    u64 p = pattern(k->code[s], k->all, rel, s);
    int n = code_len(p);
    if (total + n > 29) return;
    counts |= (u64)n << (4 * s);
    owners |= (p ^ (1ull << (2 * n))) << (2 * total);
    total += n;
  }
  u64 w1 = counts | owners << 16, hi = owners >> 48 << 53;
  OBucket* b = c->tt + k->bucket;
  for (int i = 0; i < 16; i++) {
    if ((b->tag[i] & ~0xF00u) != k->tag) continue;
    int way = (b->tag[i] >> 8) & 15;
    u64 e0 = b->w0[way];
    if ((e0 & QMASK) == k->q && b->w1[way] == w1 && e0 >> 53 << 53 == hi) {
      int olb = (int)(e0 >> QBITS) & 15, oub = (int)(e0 >> (QBITS + 4)) & 15, ob = (int)(e0 >> (QBITS + 8)) & 63;
      if (olb > lb) lb = olb;
      if (oub < ub) ub = oub;
      if (best < 0 && ob != 63) best = ob;
      b->w0[way] = k->q | (u64)lb << QBITS | (u64)ub << (QBITS + 4) | (u64)(best < 0 ? 63 : best) << (QBITS + 8) | hi;
      return;
    }
  }
  int way = tt_slot(c, b, k->tag);
  b->w0[way] = k->q | (u64)lb << QBITS | (u64)ub << (QBITS + 4) | (u64)(best < 0 ? 63 : best) << (QBITS + 8) | hi;
  b->w1[way] = w1;
}

/* src/dd.h:864-874. */
static void next_gen(OCtx* c) {
  c->gen++;
  if (c->gen >= 64) {
    for (u32 i = 0; i <= c->mask; i++) memset(c->tt[i].tag, 0, sizeof(c->tt[i].tag));
    c->gen = 1;
  }
}

/* ---- bounds (src/dd_bounds.h:11-584; DDS quick_tricks.cpp / later_tricks.cpp) --------- */

typedef struct {
  int len[4][4];
  int win_h[4], win_c[4], sec_h[4], sec_c[4], thr_h[4], thr_c[4];
} OTop;

static void top_init(OTop* t, const u64* h) {
  for (int p = 0; p < 4; p++)
    for (int s = 0; s < 4; s++) t->len[p][s] = popc(h[p] & suit_mask(s));
  for (int s = 0; s < 4; s++) {
    int hs[3] = {-1, -1, -1}, cs[3] = {0, 0, 0}, k = 0;
    for (int r = 12; r >= 0 && k < 3; r--) {
      int card = s * 16 + r;
      for (int p = 0; p < 4; p++)
        if (h[p] >> card & 1) {
          hs[k] = p;
          cs[k] = card;
          k++;
        }
    }
    t->win_h[s] = hs[0];
    t->win_c[s] = cs[0];
    t->sec_h[s] = hs[1];
    t->sec_c[s] = cs[1];
    t->thr_h[s] = hs[2];
    t->thr_c[s] = cs[2];
  }
}

static int qt_next(int suit, int trump) {
  if (trump >= 0 && suit == trump) return trump == 0 ? 1 : 0;
  suit++;
  if (trump >= 0 && suit == trump) suit++;
  return suit;
}

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

/* res: 0 stay in suit, 1 cutoff reached, 2 next suit. */
static int qt_lead_trump(const OTop* t, int hand, int cutoff, int lho, int rho, int lhoT, int rhoT,
                         int own, int part, int suit, int qt, u64* wr, int* res) {
  *res = 1;
  if ((lho != 0 || lhoT == 0) && (rho != 0 || rhoT == 0)) {
    *wr |= bitc(t->win_c[suit]);
    if (++qt >= cutoff) return qt;
    if (lho <= 1 && rho <= 1 && part <= 1 && lhoT == 0 && rhoT == 0) {
      qt += own - 1;
      if (qt >= cutoff) return qt;
      *res = 2;
      return qt;
    }
  }
  if (t->sec_h[suit] == hand) {
    if (lhoT == 0 && rhoT == 0) {
      *wr |= bitc(t->sec_c[suit]);
      if (++qt >= cutoff) return qt;
      if (lho <= 2 && rho <= 2 && part <= 2) {
        qt += own - 2;
        if (qt >= cutoff) return qt;
        *res = 2;
        return qt;
      }
    }
  } else if (t->sec_h[suit] == P_of(hand) && own > 1 && part > 1) {
    if (lhoT == 0 && rhoT == 0) {
      *wr |= bitc(t->sec_c[suit]);
      if (++qt >= cutoff) return qt;
      if (lho <= 2 && rho <= 2 && (part <= 2 || own <= 2)) {
        qt += imax(own, part) - 2;
        if (qt >= cutoff) return qt;
        *res = 2;
        return qt;
      }
    }
  }
  *res = 0;
  return qt;
}

static void qt_draw(int* lhoT, int* rhoT) {
  *lhoT = *lhoT > 0 ? *lhoT - 1 : 0;
  *rhoT = *rhoT > 0 ? *rhoT - 1 : 0;
}

static int qt_lead_nt(const OTop* t, int hand, int cutoff, int lho, int rho, int* lhoT, int* rhoT,
                      int comm, int comm_suit, int own, int part, int suit, int qt, int trump, u64* wr,
                      int* res) {
  int draws = trump == suit && (!comm || suit != comm_suit);
  *res = 1;
  *wr |= bitc(t->win_c[suit]);
  if (++qt >= cutoff) return qt;
  if (draws) qt_draw(lhoT, rhoT);
  if (lho <= 1 && rho <= 1 && part <= 1) {
    qt += own - 1;
    if (qt >= cutoff) return qt;
    *res = 2;
    return qt;
  }
  if (t->sec_h[suit] == hand) {
    *wr |= bitc(t->sec_c[suit]);
    if (++qt >= cutoff) return qt;
    if (draws) qt_draw(lhoT, rhoT);
    if (lho <= 2 && rho <= 2 && part <= 2) {
      qt += own - 2;
      if (qt >= cutoff) return qt;
      *res = 2;
      return qt;
    }
  } else if (t->sec_h[suit] == P_of(hand) && own > 1 && part > 1) {
    *wr |= bitc(t->sec_c[suit]);
    if (++qt >= cutoff) return qt;
    if (draws) qt_draw(lhoT, rhoT);
    if (lho <= 2 && rho <= 2 && (part <= 2 || own <= 2)) {
      qt += imax(own, part) - 2;
      if (qt >= cutoff) return qt;
      *res = 2;
      return qt;
    }
  }
  *res = 0;
  return qt;
}

static int qt_partner_trump(const OTop* t, int hand, int cutoff, int lho, int rho, int lhoT, int rhoT,
                            int own, int part, int suit, int qt, int comm_suit, int comm_card, u64* wr,
                            int* res) {
  int P = P_of(hand);
  *res = 1;
  if ((lho != 0 || lhoT == 0) && (rho != 0 || rhoT == 0)) {
    *wr |= bitc(t->win_c[suit]) | bitc(comm_card);
    if (++qt >= cutoff) return qt;
    if (lho <= 1 && rho <= 1 && own <= 1 && lhoT == 0 && rhoT == 0) {
      qt += part - 1;
      if (qt >= cutoff) return qt;
      *res = 2;
      return qt;
    }
  }
  if (t->sec_h[suit] == P) {
    if (lhoT == 0 && rhoT == 0) {
      *wr |= bitc(t->sec_c[suit]) | bitc(comm_card);
      if (++qt >= cutoff) return qt;
      if (lho <= 2 && rho <= 2 && own <= 2) {
        qt += part - 2;
        if (qt >= cutoff) return qt;
        *res = 2;
        return qt;
      }
    }
  } else if (t->sec_h[suit] == hand && part > 1 && own > 1) {
    if (lhoT == 0 && rhoT == 0) {
      *wr |= bitc(t->sec_c[suit]) | bitc(comm_card);
      if (++qt >= cutoff) return qt;
      if (lho <= 2 && rho <= 2 && (own <= 2 || part <= 2)) {
        qt += imax(part, own) - 2;
        if (qt >= cutoff) return qt;
        *res = 2;
        return qt;
      }
    }
  } else if (suit == comm_suit && t->sec_h[suit] == L_of(hand) && (lho >= 2 || lhoT == 0) &&
             (rho >= 2 || rhoT == 0)) {
    if (t->thr_h[suit] == P) {
      *wr |= bitc(t->thr_c[suit]) | bitc(comm_card);
      if (++qt >= cutoff) return qt;
      if (own <= 2 && lho <= 2 && rho <= 2 && lhoT == 0 && rhoT == 0) {
        qt += part - 2;
        if (qt >= cutoff) return qt;
      }
    }
  }
  *res = 0;
  return qt;
}

static int qt_partner_nt(const OTop* t, int hand, int cutoff, int lho, int rho, int own, int part,
                         int suit, int qt, int comm_suit, int comm_card, u64* wr, int* res) {
  int P = P_of(hand);
  *res = 1;
  *wr |= bitc(t->win_c[suit]) | bitc(comm_card);
  if (++qt >= cutoff) return qt;
  if (lho <= 1 && rho <= 1 && own <= 1) {
    qt += part - 1;
    if (qt >= cutoff) return qt;
    *res = 2;
    return qt;
  }
  if (t->sec_h[suit] == P) {
    *wr |= bitc(t->sec_c[suit]);
    if (++qt >= cutoff) return qt;
    if (lho <= 2 && rho <= 2 && own <= 2) {
      qt += part - 2;
      if (qt >= cutoff) return qt;
      *res = 2;
      return qt;
    }
  } else if (t->sec_h[suit] == hand && part > 1 && own > 1) {
    *wr |= bitc(t->sec_c[suit]);
    if (++qt >= cutoff) return qt;
    if (lho <= 2 && rho <= 2 && (own <= 2 || part <= 2)) {
      qt += imax(part, own) - 2;
      if (qt >= cutoff) return qt;
      *res = 2;
      return qt;
    }
  } else if (suit == comm_suit && t->sec_h[suit] == L_of(hand)) {
    if (t->thr_h[suit] == P) {
      *wr |= bitc(t->thr_c[suit]);
      if (++qt >= cutoff) return qt;
      if (own <= 2 && lho <= 2 && rho <= 2) {
        qt += part - 2;
        if (qt >= cutoff) return qt;
      }
    }
  }
  *res = 0;
  return qt;
}

/* DDS QuickTricks for the hand on lead (src/dd_bounds.h:245-438). */
static int quick_tricks(const u64* hands, const OTop* t, int trump, int hand, int cutoff, int cutoff_other,
                        u64* wr, int* decided) {
  int P = P_of(hand), L = L_of(hand), R = R_of(hand);
  int comm_card = 0, comm_suit = -1, lowest_q = 0, qtricks = 0, comm = 0;
  *decided = 1;
  for (int s = 0; s < 4; s++) {
    if (trump >= 0 && trump != s) {
      if (t->win_h[s] == P) {
        if (t->len[hand][s] != 0 && (t->len[L][s] != 0 || t->len[L][trump] == 0) &&
            (t->len[R][s] != 0 || t->len[R][trump] == 0)) {
          comm = 1, comm_suit = s, comm_card = t->win_c[s];
          break;
        }
      } else if (t->sec_h[s] == P && t->win_h[s] == hand && t->len[hand][s] >= 2 && t->len[P][s] >= 2) {
        if ((t->len[L][s] != 0 || t->len[L][trump] == 0) && (t->len[R][s] != 0 || t->len[R][trump] == 0)) {
          comm = 1, comm_suit = s, comm_card = t->sec_c[s];
          break;
        }
      }
    } else if (trump < 0) {
      if (t->win_h[s] == P) {
        if (t->len[hand][s] != 0) {
          comm = 1, comm_suit = s, comm_card = t->win_c[s];
          break;
        }
      } else if (t->sec_h[s] == P && t->win_h[s] == hand && t->len[hand][s] >= 2 && t->len[P][s] >= 2) {
        comm = 1, comm_suit = s, comm_card = t->sec_c[s];
        break;
      }
    }
  }
  if (trump >= 0 && !comm && t->len[hand][trump] != 0 && t->win_h[trump] == P)
    comm = 1, comm_suit = trump, comm_card = t->win_c[trump];

  int lhoT = 0, rhoT = 0, suit = 0;
  if (trump >= 0) {
    suit = trump;
    lhoT = t->len[L][trump];
    rhoT = t->len[R][trump];
  }
  do {
    int own = t->len[hand][suit], lho = t->len[L][suit], rho = t->len[R][suit], part = t->len[P][suit];
    int opps = lho | rho;
    if (!opps && part == 0) {
      if (own == 0) {
        suit = qt_next(suit, trump);
        continue;
      }
      if (trump >= 0 && trump != suit) {
        if (lhoT == 0 && rhoT == 0) {
          qtricks += own;
          if (qtricks >= cutoff) return qtricks;
        }
        suit = qt_next(suit, trump);
        continue;
      }
      qtricks += own;
      if (qtricks >= cutoff) return qtricks;
      suit = qt_next(suit, trump);
      continue;
    } else {
      if (!opps && trump >= 0 && suit == trump) {
        int sum = imax(own, part);
        for (int s = 0; s < 4; s++)
          if (sum > 0 && s != trump && own >= part && t->len[hand][s] > 0 && t->len[P][s] == 0) {
            sum++;
            break;
          }
        if (sum >= cutoff) return sum;
      } else if (!opps) {
        int sum = imin(own, part);
        if (trump < 0) {
          if (sum >= cutoff) return sum;
        } else if (suit != trump && lhoT == 0 && rhoT == 0) {
          if (sum >= cutoff) return sum;
        }
      }
      if (comm) {
        if (!opps && own == 0) {
          if (trump >= 0 && trump != suit) {
            if (lhoT == 0 && rhoT == 0) {
              qtricks += part;
              *wr |= bitc(comm_card);
              if (qtricks >= cutoff) return qtricks;
            }
            suit = qt_next(suit, trump);
            continue;
          }
          qtricks += part;
          *wr |= bitc(comm_card);
          if (qtricks >= cutoff) return qtricks;
          suit = qt_next(suit, trump);
          continue;
        } else if (!opps && trump >= 0 && suit == trump) {
          int sum = imax(own, part);
          for (int s = 0; s < 4; s++)
            if (sum > 0 && s != trump && own <= part && t->len[P][s] > 0 && t->len[hand][s] == 0) {
              sum++;
              break;
            }
          if (sum >= cutoff) {
            *wr |= bitc(comm_card);
            return sum;
          }
        } else if (!opps) {
          int sum = imin(own, part);
          if (trump < 0) {
            if (sum >= cutoff) return sum;
          } else if (suit != trump && lhoT == 0 && rhoT == 0) {
            if (sum >= cutoff) return sum;
          }
        }
      }
    }
    if (t->win_h[suit] < 0) {
      suit = qt_next(suit, trump);
      continue;
    }
    int res;
    if (t->win_h[suit] == hand) {
      if (trump >= 0 && trump != suit)
        qtricks = qt_lead_trump(t, hand, cutoff, lho, rho, lhoT, rhoT, own, part, suit, qtricks, wr, &res);
      else
        qtricks = qt_lead_nt(t, hand, cutoff, lho, rho, &lhoT, &rhoT, comm, comm_suit, own, part, suit,
                             qtricks, trump, wr, &res);
      if (res == 1) return qtricks;
      if (res == 2) {
        suit = qt_next(suit, trump);
        continue;
      }
    } else if (t->win_h[suit] == P && comm) {
      if (trump >= 0 && trump != suit)
        qtricks = qt_partner_trump(t, hand, cutoff, lho, rho, lhoT, rhoT, own, part, suit, qtricks,
                                   comm_suit, comm_card, wr, &res);
      else
        qtricks = qt_partner_nt(t, hand, cutoff, lho, rho, own, part, suit, qtricks, comm_suit, comm_card,
                                wr, &res);
      if (res == 1) return qtricks;
      if (res == 2) {
        suit = qt_next(suit, trump);
        continue;
      }
    }
    if (trump >= 0 && suit != trump && own > 0 && lowest_q == 0 &&
        (qtricks == 0 || (t->win_h[suit] != hand && t->win_h[suit] != P && t->win_h[trump] != hand &&
                          t->win_h[trump] != P))) {
      u64 T = suit_mask(trump), pt = hands[P] & T;
      if (part == 0 && t->len[P][trump] > 0) {
        if ((rho > 0 || t->len[R][trump] == 0) && (lho > 0 || t->len[L][trump] == 0)) {
          lowest_q = 1;
          if (1 >= cutoff) return 1;
          suit = qt_next(suit, trump);
          continue;
        }
        u64 over = 0;
        if (rho == 0 && lho == 0) over = (hands[L] | hands[R]) & T;
        else if (lho == 0) over = hands[L] & T;
        else over = hands[R] & T;
        if (over < pt) {
          lowest_q = 1;
          *wr |= bitc(msb(pt));
          if (1 >= cutoff) return 1;
        }
        suit = qt_next(suit, trump);
        continue;
      }
    }
    if (qtricks >= cutoff) return qtricks;
    suit = qt_next(suit, trump);
  } while (suit <= 3);

  if (qtricks == 0 && (trump < 0 || t->win_h[trump] < 0)) {
    for (int s = 0; s < 4; s++) {
      if (t->win_h[s] < 0) continue;
      if (t->len[hand][s] > 0) *wr = (*wr & ~suit_mask(s)) | bitc(t->win_c[s]);
    }
    if (1 >= cutoff_other) return 0;
  }
  *decided = 0;
  return qtricks;
}

/* DDS QuickTricksSecondHand (src/dd_bounds.h:442-479). */
static int quick_tricks_2nd(const u64* hands, const OTop* t, int trump, int hand, int lead, int cutoff,
                            u64* wr) {
  int ss = lead >> 4, P = P_of(hand), L = L_of(hand);
  u64 S = suit_mask(ss), T = trump >= 0 ? suit_mask(trump) : 0;
  u64 ranks = (hands[hand] | hands[P]) & S;
  *wr = 0;
  if (trump >= 0 && ss != trump &&
      ((!(hands[hand] & S) && (hands[hand] & T)) || (!(hands[P] & S) && (hands[P] & T)))) {
    if (!(hands[L] & S) && (hands[L] & T)) return 0;
  } else if (ranks > (bitc(lead) | (hands[L] & S))) {
    if (trump >= 0 && ss != trump && (hands[L] & T) && !(hands[L] & S)) return 0;
    *wr = bitc(msb(ranks));
  } else {
    return 0;
  }
  int qtricks = 1;
  if (qtricks >= cutoff) return 1;
  if (trump >= 0) return 0;
  int hh = (hands[hand] & S) > (hands[P] & S) ? hand : P;
  if (t->win_h[ss] == hh && t->sec_h[ss] == hh) {
    qtricks++;
    *wr |= bitc(t->sec_c[ss]);
    if (qtricks >= cutoff) return 1;
  }
  for (int s = 0; s < 4; s++) {
    if (s == ss || !(hands[hh] & suit_mask(s))) continue;
    if (!((hands[L_of(hh)] | hands[R_of(hh)] | hands[P_of(hh)]) & suit_mask(s))) {
      qtricks += popc(hands[hh] & suit_mask(s));
      if (qtricks >= cutoff) return 1;
    } else if (t->win_h[s] == hh) {
      qtricks++;
      *wr |= bitc(t->win_c[s]);
      if (qtricks >= cutoff) return 1;
    }
  }
  return 0;
}

/* DDS LaterTricksMIN (src/dd_bounds.h:482-531). 0 = NS cannot reach target. */
static int later_min(const OTop* t, int trump, int hand, int ns_won, int left, int target, u64* wr) {
  int dq = left - 1;
  if (trump < 0 || t->win_h[trump] < 0) {
    int sum = 0;
    for (int s = 0; s < 4; s++) {
      int hh = t->win_h[s];
      if (hh >= 0 && is_ns(hh)) sum += imax(t->len[hh][s], t->len[P_of(hh)][s]);
    }
    if (ns_won + sum < target && sum > 0) {
      if (ns_won + dq >= target) return 1;
      *wr = 0;
      for (int s = 0; s < 4; s++) {
        int wh = t->win_h[s];
        if (wh >= 0 && !is_ns(wh) && (t->len[P_of(wh)][s] || t->len[L_of(wh)][s] || t->len[R_of(wh)][s]))
          *wr |= bitc(t->win_c[s]);
      }
      return 0;
    }
  } else if (!is_ns(t->win_h[trump])) {
    if (t->len[hand][trump] == 0 && t->len[P_of(hand)][trump] == 0) {
      int m = imax(t->len[L_of(hand)][trump], t->len[R_of(hand)][trump]);
      if (ns_won + dq + 1 - m < target) {
        *wr = 0;
        return 0;
      }
    } else if (ns_won + dq < target) {
      *wr = bitc(t->win_c[trump]);
      return 0;
    } else if (ns_won + dq == target) {
      int hh = t->sec_h[trump];
      if (hh < 0) return 1;
      if (!is_ns(hh) && (t->len[hh][trump] > 1 || t->len[P_of(hh)][trump] > 1)) {
        *wr = bitc(t->sec_c[trump]);
        return 0;
      }
    }
  } else {
    int hh = t->sec_h[trump];
    if (hh < 0) return 1;
    if (is_ns(hh) || t->len[hh][trump] <= 1) return 1;
    if (t->win_h[trump] == R_of(hh)) {
      if (ns_won + dq < target) {
        *wr = bitc(t->sec_c[trump]);
        return 0;
      }
    } else {
      int h3 = t->thr_h[trump];
      if (h3 < 0) return 1;
      if (!is_ns(h3) && ns_won + dq < target) {
        *wr = bitc(t->thr_c[trump]);
        return 0;
      }
    }
  }
  return 1;
}

/* DDS LaterTricksMAX (src/dd_bounds.h:534-584). 1 = NS reach target. */
static int later_max(const OTop* t, int trump, int hand, int ns_won, int left, int target, u64* wr) {
  int dq = left - 1;
  if (trump < 0 || t->win_h[trump] < 0) {
    int sum = 0;
    for (int s = 0; s < 4; s++) {
      int hh = t->win_h[s];
      if (hh >= 0 && !is_ns(hh)) sum += imax(t->len[hh][s], t->len[P_of(hh)][s]);
    }
    if (ns_won + dq + 1 - sum >= target && sum > 0) {
      if (ns_won + 1 < target) return 0;
      *wr = 0;
      for (int s = 0; s < 4; s++) {
        int wh = t->win_h[s];
        if (wh >= 0 && is_ns(wh) && (t->len[P_of(wh)][s] || t->len[L_of(wh)][s] || t->len[R_of(wh)][s]))
          *wr |= bitc(t->win_c[s]);
      }
      return 1;
    }
  } else if (is_ns(t->win_h[trump])) {
    if (t->len[hand][trump] == 0 && t->len[P_of(hand)][trump] == 0) {
      int m = imax(t->len[L_of(hand)][trump], t->len[R_of(hand)][trump]);
      if (ns_won + m >= target) {
        *wr = 0;
        return 1;
      }
    } else if (ns_won + 1 >= target) {
      *wr = bitc(t->win_c[trump]);
      return 1;
    } else {
      int hh = t->sec_h[trump];
      if (hh < 0) return 0;
      if (is_ns(hh) && (t->len[hh][trump] > 1 || t->len[P_of(hh)][trump] > 1) && ns_won + 2 >= target) {
        *wr = bitc(t->sec_c[trump]);
        return 1;
      }
    }
  } else {
    int hh = t->sec_h[trump];
    if (hh < 0) return 0;
    if (!is_ns(hh) || t->len[hh][trump] <= 1) return 0;
    if (t->win_h[trump] == R_of(hh)) {
      if (ns_won + 1 >= target) {
        *wr = bitc(t->sec_c[trump]);
        return 1;
      }
    } else {
      int h3 = t->thr_h[trump];
      if (h3 < 0) return 0;
      if (is_ns(h3) && ns_won + 1 >= target) {
        *wr = bitc(t->thr_c[trump]);
        return 1;
      }
    }
  }
  return 0;
}

/* ---- move ordering (src/dd_bounds.h:586-949; DDS heuristic_sorting.cpp) ------------- */

static int R2(int card) { return (card & 15) + 2; }
static int hi2(u64 m) { return m ? (msb(m) & 15) + 2 : 0; }
static int lo2(u64 m) { return m ? (lsb(m) & 15) + 2 : 0; }

/* Cards of the suit at or above `card`, among those in play (1 = highest). */
static int rank_from_top(u64 all, int card) {
  int s = card >> 4, n = 0;
  for (int r = card & 15; r < 13; r++) n += (int)(all >> (s * 16 + r) & 1);
  return n;
}
/* Is the next lower card in play (in `all`) of the suit held by `own`? */
static int next_lower_is(u64 all, u64 own, int card) {
  int s = card >> 4;
  for (int r = (card & 15) - 1; r >= 0; r--)
    if (all >> (s * 16 + r) & 1) return (int)(own >> (s * 16 + r) & 1);
  return 0;
}

static int lead_weight(const u64* hands, const OTop* t, int trump, int left, int lead, int card, int tt) {
  int s = card >> 4, P = P_of(lead), L = L_of(lead), R = R_of(lead);
  u64 S = suit_mask(s), all = hands[0] | hands[1] | hands[2] | hands[3];
  int r_rank = rank_from_top(all, card);
  int seq = next_lower_is(all, hands[lead], card);
  u64 risP = hands[P] & S, risL = hands[L] & S, risR = hands[R] & S;
  int cntLH = (t->len[L][s] == 0 ? left : t->len[L][s]) << 2;
  int cntRH = (t->len[R][s] == 0 ? left : t->len[R][s]) << 2;
  int w;
  if (trump >= 0 && (all & suit_mask(trump))) {
    u64 T = suit_mask(trump);
    int bonus = 0, win = 0;
    if (s != trump && ((!risL && (hands[L] & T)) || (!risR && (hands[R] & T)))) bonus = -12;
    if (s != trump && t->len[P][s] == 0 && t->len[P][trump] > 0 && t->len[R][s] > 0) bonus += 17;
    if (t->win_h[s] == R || t->sec_h[s] == R) {
      if (t->len[R][s] != 1) bonus += -12;
    } else if (t->win_h[s] == L && t->sec_h[s] == P) {
      if (t->len[P][s] != 1) bonus += 27;
    }
    if (s != trump && t->len[lead][s] == 1 && t->len[lead][trump] > 0 && t->len[P][s] > 1 && t->win_h[s] == P)
      bonus += 19;
    int delta = bonus - (((cntLH + cntRH) << 5) / 13);
    if (t->win_c[s] == card) {
      if (s != trump) {
        if (t->len[P][s] != 0 || t->len[P][trump] == 0) {
          if ((t->len[L][s] != 0 || t->len[L][trump] == 0) && (t->len[R][s] != 0 || t->len[R][trump] == 0))
            win = 1;
        } else if ((t->len[L][s] != 0 || (hands[P] & T) > (hands[L] & T)) &&
                   (t->len[R][s] != 0 || (hands[P] & T) > (hands[R] & T))) {
          win = 1;
        }
      } else {
        win = 1;
      }
    } else if (risP > (risL | risR)) {
      if (s != trump) {
        if ((t->len[L][s] != 0 || t->len[L][trump] == 0) && (t->len[R][s] != 0 || t->len[R][trump] == 0))
          win = 1;
      } else {
        win = 1;
      }
    } else if (s != trump) {
      if (t->len[P][s] == 0 && t->len[P][trump] != 0) {
        if (t->len[L][s] == 0 && t->len[L][trump] != 0 && t->len[R][s] == 0 && t->len[R][trump] != 0) {
          if ((hands[P] & T) > ((hands[L] | hands[R]) & T)) win = 1;
        } else if (t->len[L][s] == 0 && t->len[L][trump] != 0) {
          if ((hands[P] & T) > (hands[L] & T)) win = 1;
        } else if (t->len[R][s] == 0 && t->len[R][trump] != 0) {
          if ((hands[P] & T) > (hands[R] & T)) win = 1;
        } else {
          win = 1;
        }
      }
    }
    if (win) {
      if ((t->len[L][s] == 1 && t->win_h[s] == L) || (t->len[R][s] == 1 && t->win_h[s] == R))
        w = delta + 35 + r_rank;
      else if (t->win_h[s] == lead) {
        if (t->sec_h[s] == P) w = delta + 48 + r_rank;
        else if (t->win_c[s] == card) w = delta + 31;
        else w = delta - 3 + r_rank;
      } else if (t->win_h[s] == P) {
        w = delta + (t->sec_h[s] == lead ? 42 : 28) + r_rank;
      } else if (seq && card == t->sec_c[s]) {
        w = delta + 40;
      } else if (seq) {
        w = delta + 22 + r_rank;
      } else {
        w = delta + 11 + r_rank;
      }
      if (tt) w += 18;
    } else {
      int third = t->thr_h[s];
      if (t->sec_h[s] == P && P == third) delta += 20;
      else if ((t->sec_h[s] == lead && P == third && t->len[P][s] > 1) ||
               (t->sec_h[s] == P && lead == third && t->len[P][s] > 1))
        delta += 13;
      if ((t->len[L][s] == 1 && t->win_h[s] == L) || (t->len[R][s] == 1 && t->win_h[s] == R))
        w = delta + r_rank + 2;
      else if (t->win_h[s] == lead) {
        if (t->sec_h[s] == P) w = delta + 33 + r_rank;
        else if (t->win_c[s] == card) w = delta + 38;
        else w = delta - 14 + r_rank;
      } else if (t->win_h[s] == P) {
        w = delta + 34 + r_rank;
      } else if (seq && card == t->sec_c[s]) {
        w = delta + 35;
      } else {
        w = delta + 17 - R2(card);
      }
    }
    return w;
  }
  int delta = -(((cntLH + cntRH) << 5) / 19);
  if (t->len[P][s] == 0) delta += -9;
  if (t->win_c[s] == card || risP > (risL | risR)) {
    if (t->sec_h[s] == R) {
      if (t->len[R][s] != 1) delta += -1;
    } else if (t->sec_h[s] == L) {
      delta += t->len[L][s] != 1 ? 22 : 16;
    }
    if ((t->sec_h[s] != L || t->len[L][s] == 1) && (t->sec_h[s] != R || t->len[R][s] == 1))
      w = delta + 45 + r_rank;
    else
      w = delta + 18 + r_rank;
    if (tt) w += 32;
  } else {
    if (t->win_h[s] == R || t->sec_h[s] == R) {
      if (t->len[R][s] != 1) delta += -10;
    } else if (t->win_h[s] == L && t->sec_h[s] == P) {
      if (t->len[P][s] != 1) delta += 31;
    }
    int third = t->thr_h[s];
    if (t->sec_h[s] == P && P == third) delta += 35;
    else if ((t->sec_h[s] == lead && P == third && t->len[P][s] > 1) ||
             (t->sec_h[s] == P && lead == third && t->len[P][s] > 1))
      delta += 25;
    if ((t->len[L][s] == 1 && t->win_h[s] == L) || (t->len[R][s] == 1 && t->win_h[s] == R))
      w = delta + 28 + r_rank;
    else if (t->win_h[s] == lead) w = delta - 17 + r_rank;
    else if (!seq) w = delta + 12 + r_rank;
    else if (card == t->sec_c[s]) w = delta + 48;
    else w = delta + 29 - r_rank;
    if (tt) w += 19;
  }
  return w;
}

static int beats(int card, int best, int trump) {
  int s = card >> 4, bs = best >> 4;
  if (s == bs) return card > best;
  return s == trump;
}

typedef struct {
  u64 th[4], allt, all;
  int win_h[4], sec_h[4];
  int lead, ls, lead0, P, R, high1, high2, move1, move2;
} OFollow;

static void follow_init(OFollow* f, const u64* hands, int trump, int leader, const int* trick, int n) {
  f->lead = leader;
  f->ls = trick[0] >> 4;
  f->P = P_of(leader);
  f->R = R_of(leader);
  for (int h = 0; h < 4; h++) f->th[h] = hands[h];
  for (int i = 0; i < n; i++) f->th[(leader + i) & 3] |= bitc(trick[i]);
  f->all = hands[0] | hands[1] | hands[2] | hands[3];
  f->allt = f->th[0] | f->th[1] | f->th[2] | f->th[3];
  for (int s = 0; s < 4; s++) {
    int k = 0;
    f->win_h[s] = f->sec_h[s] = -1;
    for (int r = 12; r >= 0 && k < 2; r--) {
      int card = s * 16 + r;
      if (f->allt >> card & 1) {
        int o = owner(f->th, card);
        if (k == 0) f->win_h[s] = o;
        else f->sec_h[s] = o;
        k++;
      }
    }
  }
  f->lead0 = R2(trick[0]);
  int w1 = n > 1 && beats(trick[1], trick[0], trump) ? 1 : 0;
  int w2 = n > 2 && beats(trick[2], trick[w1], trump) ? 2 : w1;
  f->high1 = w1;
  f->move1 = trick[w1];
  f->high2 = w2;
  f->move2 = trick[w2];
}

static int follow_weight(const OFollow* f, const u64* hands, int trump, int n, int seat, int card) {
  int lead = f->lead, ls = f->ls, s = card >> 4, rank = R2(card), P = f->P, R = f->R;
  u64 LS = suit_mask(ls), T = trump >= 0 ? suit_mask(trump) : 0;
  int r_rank = rank_from_top(f->all, card);
  int seq = next_lower_is(f->allt, hands[seat], card);
  int lead0 = f->lead0, is_void = s != ls;
  int sc = popc(hands[seat] & suit_mask(s));
  int sec_mine = f->sec_h[s] == seat, win_mine = f->win_h[s] == seat;
  if (n == 1) {
    int max3rd = hi2(hands[P] & LS), maxpd = hi2(hands[R] & LS);
    int min3rd = lo2(hands[P] & LS), minpd = lo2(hands[R] & LS);
    if (!is_void) {
      if (trump >= 0) {
        int win = 0;
        if (ls == trump) {
          if (maxpd > lead0 && maxpd > max3rd) win = 1;
          else if (rank > lead0 && rank > max3rd) win = 1;
        } else if (rank > lead0 && rank > max3rd) {
          if (max3rd != 0 || !(hands[P] & T)) win = 1;
          else if (maxpd == 0 && (hands[R] & T) && (hands[R] & T) > (hands[P] & T)) win = 1;
        } else if (maxpd > lead0 && maxpd > max3rd) {
          if (max3rd != 0 || !(hands[P] & T)) win = 1;
        } else if (lead0 > maxpd && lead0 > max3rd && lead0 > rank) {
          if (maxpd == 0 && (hands[R] & T)) {
            if (max3rd != 0 || !(hands[P] & T)) win = 1;
            else if ((hands[R] & T) > (hands[P] & T)) win = 1;
          }
        } else if (maxpd == 0 && (hands[R] & T)) {
          win = 1;
        }
        if (win) {
          if (min3rd > rank) return 40 + r_rank;
          if (maxpd > lead0 && (hands[lead] & LS) > (hands[R] & LS)) return 41 + r_rank;
          if (rank > lead0) {
            if (rank < maxpd) return 78 - rank;
            if (rank > max3rd) return 73 - rank;
            if (seq) return 62 - rank;
            return 49 - rank;
          }
          return maxpd > 0 ? 47 - rank : 40 - rank;
        }
        if (rank < min3rd || rank < minpd) return -9 + r_rank;
        if (rank < lead0) return -16 + r_rank;
        return seq ? 22 - rank : 10 - rank;
      }
      if (maxpd > lead0 && maxpd > max3rd) return -rank;
      if (rank > lead0 && rank > max3rd) return 81 - rank;
      if (min3rd > rank || minpd > rank) return -3 + r_rank;
      if (rank < lead0) return -11 + r_rank;
      return seq ? 10 + r_rank : 13 - rank;
    }
    u64 lead_bit = bitc((ls << 4) | (lead0 - 2));
    int add;
    if (trump >= 0) {
      if (ls == trump) {
        if ((hands[R] & LS) > ((hands[P] & LS) | lead_bit)) add = (sc << 6) / 44;
        else {
          add = (sc << 6) / 36;
          if (sc == 2 && sec_mine) add += -4;
        }
        return -rank + add;
      }
      if (s != trump) {
        if (hands[P] & LS) {
          if ((hands[R] & LS) > ((hands[P] & LS) | lead_bit)) add = 60 + (sc << 6) / 44;
          else if (!(hands[R] & LS) && (hands[R] & T)) add = 60 + (sc << 6) / 44;
          else {
            add = -2 + (sc << 6) / 36;
            if (sc == 2 && sec_mine) add += -4;
          }
        } else if (!(hands[R] & LS) && (hands[R] & T) > (hands[P] & T)) {
          add = 60 + (sc << 6) / 44;
        } else if (!(hands[P] & T) && (hands[R] & LS) > lead_bit) {
          add = 60 + (sc << 6) / 44;
        } else {
          add = -2 + (sc << 6) / 36;
          if (sc == 2 && sec_mine) add += -4;
        }
        return -rank + add;
      }
      if ((hands[P] & LS) || (!(hands[R] & LS) && (hands[R] & T) && (hands[R] & T) > (hands[P] & T)))
        return 24 - rank + (sc << 6) / 44;
      if (bitc(card) > (hands[P] & T)) return 24 - rank + (sc << 6) / 44;
      add = (sc << 6) / 36;
      if (sc == 2 && sec_mine) add += -4;
      return 15 - rank + add;
    }
    if ((hands[R] & LS) > ((hands[P] & LS) | lead_bit)) {
      add = (sc << 6) / 23;
      if (sc == 2 && sec_mine) add += -2;
      else if (sc == 1 && win_mine) add += -3;
    } else {
      add = (sc << 6) / 33;
      if (sc == 2 && sec_mine) add += -6;
      else if (sc == 1 && win_mine) add += -8;
    }
    return -rank + add;
  }
  if (n == 2) {
    u64 c4 = hands[R] & LS;
    int max4th = hi2(c4), min4th = lo2(c4), m1r = R2(f->move1), m1s = f->move1 >> 4;
    if (!is_void) {
      int max3rd = hi2(hands[seat] & LS);
      if (trump >= 0) {
        if (ls == trump) {
          if (f->high1 == 0 && lead0 > max4th) return -rank;
          if (max3rd < min4th || max3rd < m1r) return -rank;
          if (max3rd > max4th) return rank > max4th && rank > m1r ? 58 - rank : -rank;
          return -rank;
        }
        if (m1s == trump) return -rank;
        if (f->high1 == 0) {
          if (max4th == 0 || lead0 > max4th) return -rank;
          if (max3rd < min4th || max3rd < m1r) return -rank;
          if (max3rd > max4th) return rank > max4th ? 58 - rank : -rank;
          return rank > m1r && rank > max4th ? 60 - rank : -rank;
        }
        if (max4th == 0) return rank > m1r ? 20 - rank : -rank;
        if (max3rd < min4th || max3rd < m1r) return -rank;
        if (max3rd > max4th) return rank > m1r && rank > max4th ? 58 - rank : -rank;
        return rank > m1r && rank > max4th ? 60 - rank : -rank;
      }
      if (f->high1 == 0 && lead0 > max4th) return -rank;
      if (max3rd < min4th || max3rd < m1r) return -rank;
      return rank > m1r && rank > max4th ? 60 - rank : -rank;
    }
    if (trump >= 0) {
      if (ls == trump || s != trump) return -rank + (sc << 6) / 40;
      if (f->high1 == 0 && lead0 > max4th && (max4th != 0 || !(hands[R] & T))) return -rank - 50;
      if (m1s == trump && rank < m1r) return -32 + r_rank + (sc << 6) / 40;
      int add = (sc << 6) / 50;
      if (f->high1 == 0) {
        if (max4th != 0) return (f->sec_h[ls] == lead ? 36 : 48) - rank + add;
        if (bitc(card) > (hands[R] & T)) return 48 - rank + add;
        return -12 - rank + add;
      }
      if (max4th != 0) return 72 - rank + add;
      if (bitc(card) > (hands[R] & T)) return 48 - rank + add;
      return 36 - rank + add;
    }
    int add = (sc << 6) / 24;
    if (sc == 2 && sec_mine) add -= 4;
    if (sc == 1 && win_mine) add -= 4;
    return -rank + add;
  }
  int m2r = R2(f->move2), m2s = f->move2 >> 4;
  if (!is_void) {
    if (f->high2 == 1 || (ls != trump && m2s == trump)) return -rank;
    return rank > m2r ? 30 - rank : -rank;
  }
  if (trump >= 0) {
    int val = (sc << 6) / 24;
    if (sc == 2 && sec_mine) val -= 2;
    if (ls == trump) return -rank + val;
    if (f->high2 == 1) return s == trump ? 2 - rank + val : 25 - rank + val;
    if (m2s == trump) {
      if (s == trump) return rank > m2r ? 33 + r_rank : -13 + r_rank;
      return 14 - rank + val;
    }
    if (s == trump) return 33 + r_rank;
    return 14 - rank + val;
  }
  int val = (sc << 6) / 27;
  if (sc == 2 && sec_mine) val -= 6;
  else if (sc == 1 && win_mine) val -= 8;
  return -rank + val;
}

/* Two cards of one hand are alike: same suit and no other hand's card between them
 * (src/dd.h:554-559). */
static int equal_cards(u64 own, u64 all, int a, int b) {
  if ((a >> 4) != (b >> 4)) return 0;
  int lo = a < b ? a : b, hi = a < b ? b : a;
  for (int c = lo + 1; c < hi; c++)
    if ((all >> c & 1) && !(own >> c & 1)) return 0;
  return 1;
}

/* Candidate moves, best first (src/dd.h:562-611). A card is left out when the next higher
 * card in play of its suit is the same hand's (checked card by card). */
static int gen_moves(const OCtx* c, int seat, int hint, const OTop* t, int* out) {
  u64 own = c->hand[seat], legal = own;
  if (c->nplayed) {
    u64 f = own & suit_mask(c->trick[0] >> 4);
    if (f) legal = f;
  }
  u64 all = c->hand[0] | c->hand[1] | c->hand[2] | c->hand[3];
  for (int i = 0; i < c->nplayed; i++) all |= bitc(c->trick[i]);
  OFollow f;
  memset(&f, 0, sizeof(f));
  if (c->nplayed) follow_init(&f, c->hand, c->trump, c->leader, c->trick, c->nplayed);
  int n = 0, score[13];
  for (int card = 63; card >= 0; card--) {
    if (!(legal >> card & 1)) continue;
    int s = card >> 4, skip = 0;
    for (int r = (card & 15) + 1; r < 13; r++) {
      int up = s * 16 + r;
      if (all >> up & 1) {
        skip = (int)(own >> up & 1);
        break;
      }
    }
    if (skip) continue;
    int sc;
    int hinted = hint >= 0 && equal_cards(own, all, hint, card);
    if (c->nplayed == 0) sc = lead_weight(c->hand, t, c->trump, c->left, seat, card, hinted);
    else sc = hinted ? 1000 : follow_weight(&f, c->hand, c->trump, c->nplayed, seat, card);
    int i = n++;
    while (i > 0 && score[i - 1] < sc) {
      score[i] = score[i - 1];
      out[i] = out[i - 1];
      i--;
    }
    score[i] = sc;
    out[i] = card;
  }
  return n;
}

/* ---- search (src/dd.h:613-939) ----------------------------------------------------- */

static int winner_index(const OCtx* c) {
  int w = 0;
  for (int i = 1; i < 4; i++)
    if (beats(c->trick[i], c->trick[w], c->trump)) w = i;
  return w;
}

/* Relevance widened through the hand's own touching cards (src/dd.h:772-789). */
static u64 widen(const OCtx* c, int seat, u64 acc) {
  u64 own = c->hand[seat], all = c->hand[0] | c->hand[1] | c->hand[2] | c->hand[3];
  for (int i = 0; i < c->nplayed; i++) all |= bitc(c->trick[i]);
  for (int s = 0; s < 4; s++) {
    u64 r = acc & suit_mask(s);
    if (!r) continue;
    int low = lsb(r);
    while (own >> low & 1) {
      int next = -1;
      for (int x = low - 1; x >= s * 16; x--)
        if (all >> x & 1) {
          next = x;
          break;
        }
      if (next < 0 || !(own >> next & 1)) break;
      low = next;
      acc |= bitc(low);
    }
  }
  return acc;
}

/* Can NS take >= target tricks in total? *rel = cards whose ranks decided it. One call is
 * one node (src/dd.h:626-737, 801-862). */
static int search(OCtx* c, int target, u64* rel) {
  c->nodes++;
  int need = 0, hint = -1, lb = 0, ub = 0;
  OTop t;
  OKey key;
  if (c->nplayed == 0) {
    *rel = 0;
    if (c->ns_won >= target) return 1;
    if (c->ns_won + c->left < target) return 0;
    need = target - c->ns_won;
    u64 all = c->hand[0] | c->hand[1] | c->hand[2] | c->hand[3];
    if (c->left == 1) {
      int s = c->trump >= 0 && (all & suit_mask(c->trump)) ? c->trump : msb(c->hand[c->leader]) >> 4;
      u64 in = all & suit_mask(s);
      int top = msb(in);
      if (popc(in) >= 2) *rel = bitc(top);
      return is_ns(owner(c->hand, top));
    }
    make_key(c, &key);
    int hit = tt_probe(c, &key, need, rel, &hint);
    if (hit >= 0) return hit;
    ub = c->left;
    top_init(&t, c->hand);
    int ns_lead = is_ns(c->leader);
    int cut_ns = need, cut_ew = c->left - need + 1, decided;
    u64 wr = 0;
    int q = quick_tricks(c->hand, &t, c->trump, c->leader, ns_lead ? cut_ns : cut_ew,
                         ns_lead ? cut_ew : cut_ns, &wr, &decided);
    if (decided) {
      int val = ns_lead ? q != 0 : q == 0;
      tt_store(c, &key, wr, val ? need : 0, val ? c->left : need - 1, -1);
      *rel = wr;
      return val;
    }
    wr = 0;
    if (ns_lead ? !later_min(&t, c->trump, c->leader, c->ns_won, c->left, target, &wr)
                : later_max(&t, c->trump, c->leader, c->ns_won, c->left, target, &wr)) {
      int val = !ns_lead;
      tt_store(c, &key, wr, val ? need : 0, val ? c->left : need - 1, -1);
      *rel = wr;
      return val;
    }
  } else if (c->nplayed == 1) {
    u64 th[4] = {c->hand[0], c->hand[1], c->hand[2], c->hand[3]};
    th[c->leader] |= bitc(c->trick[0]);
    top_init(&t, th);
    int second = L_of(c->leader), need2 = target - c->ns_won;
    int cutoff = is_ns(second) ? need2 : c->left - need2 + 1;
    u64 wr;
    if (quick_tricks_2nd(c->hand, &t, c->trump, second, c->trick[0], cutoff, &wr)) {
      *rel = wr;
      return is_ns(second);
    }
  }
  int seat = (c->leader + c->nplayed) & 3, ns_turn = is_ns(seat);
  int moves[13];
  int n = gen_moves(c, seat, hint, &t, moves);
  int result = !ns_turn, best = -1;
  u64 acc = 0, tried = 0;
  for (int i = 0; i < n; i++) {
    int card = moves[i], s = card >> 4;
    u64 rs = acc & suit_mask(s);
    u64 small = rs ? (bitc(lsb(rs)) - 1) & suit_mask(s) : suit_mask(s);
    if ((small & bitc(card)) && (small & tried)) continue;
    tried |= bitc(card);
    /* play */
    int saved[4], old_leader = c->leader, win_card = -1, ended = 0;
    c->hand[seat] ^= bitc(card);
    c->trick[c->nplayed++] = card;
    if (c->nplayed == 4) {
      ended = 1;
      int wi = winner_index(c), w = (c->leader + wi) & 3, wc = c->trick[wi], same = 0;
      for (int k = 0; k < 4; k++) same += (c->trick[k] >> 4) == (wc >> 4);
      for (int k = 0; k < 4; k++) saved[k] = c->trick[k];
      win_card = same >= 2 ? wc : -1;
      c->leader = w;
      c->nplayed = 0;
      c->left--;
      c->ns_won += is_ns(w);
    }
    u64 r;
    int v = search(c, target, &r);
    /* unplay */
    if (ended) {
      for (int k = 0; k < 4; k++) c->trick[k] = saved[k];
      c->ns_won -= is_ns(c->leader);
      c->left++;
      c->nplayed = 4;
      c->leader = old_leader;
      if (win_card >= 0) r |= bitc(win_card);
    }
    c->nplayed--;
    c->hand[seat] ^= bitc(card);
    if (v == ns_turn) {
      result = v;
      acc = r;
      best = card;
      break;
    }
    acc |= r;
  }
  acc = widen(c, seat, acc);
  if (c->nplayed == 0) {
    if (result) lb = need;
    else ub = need - 1;
    tt_store(c, &key, acc, lb, ub, best);
  }
  *rel = acc;
  return result;
}

/* NS tricks with `leader` on lead: binary search from the guess (src/dd.h:877-891). */
static int ns_tricks(OCtx* c, int leader, int guess) {
  c->leader = leader;
  c->nplayed = 0;
  c->ns_won = 0;
  c->left = popc(c->hand[0]);
  int lo = 0, hi = 13, t = guess < 1 ? 1 : guess > 13 ? 13 : guess;
  u64 rel;
  while (lo < hi) {
    if (search(c, t, &rel)) lo = t;
    else hi = t - 1;
    t = (lo + hi + 1) / 2;
  }
  return lo;
}

/* Stepping from a seed (src/dd.h:898-912). */
static int ns_tricks_from(OCtx* c, int leader, int guess) {
  c->leader = leader;
  c->nplayed = 0;
  c->ns_won = 0;
  c->left = popc(c->hand[0]);
  int t = guess < 0 ? 0 : guess > c->left ? c->left : guess;
  u64 rel;
  if (t == 0 || search(c, t, &rel)) {
    while (t < c->left && search(c, t + 1, &rel)) t++;
    return t;
  }
  t--;
  while (t > 0 && !search(c, t, &rel)) t--;
  return t;
}

/* ---- C ABI ------------------------------------------------------------------------- */

typedef struct {
  OCtx c;
  OBucket* tt;
} OSolver;

static OSolver* solver_new(int tt_log2) {
  OSolver* s = (OSolver*)calloc(1, sizeof(OSolver));
  s->tt = (OBucket*)calloc((size_t)1 << tt_log2, sizeof(OBucket));
  s->c.tt = s->tt;
  s->c.mask = (1u << tt_log2) - 1;
  return s;
}
static void solver_free(OSolver* s) {
  free(s->tt);
  free(s);
}

/* One job: declarers decl0..decl1 of one strain sharing the TT; seeds = NS seeds per
 * declarer or NULL (binary search from 7, then from the previous answer). */
static void solve_job(OCtx* c, const u64* hands, int strain, int decl0, int decl1, const int8_t* seeds4,
                      int* out4) {
  for (int i = 0; i < 4; i++) c->hand[i] = hands[i];
  c->trump = strain == 4 ? -1 : 3 - strain;
  next_gen(c);
  int guess = 7;
  for (int d = decl0; d <= decl1; d++) {
    int ns = seeds4 ? ns_tricks_from(c, (d + 1) & 3, seeds4[d]) : ns_tricks(c, (d + 1) & 3, guess);
    guess = ns;
    out4[d] = (d & 1) == 0 ? ns : 13 - ns;
  }
}

typedef struct {
  const u64* hands;
  long n;
  int tt_log2, jpd;
  const int8_t* seeds;
  int* out20;
  u64* job_nodes;
  long next;
  pthread_mutex_t mu;
  u64 nodes;
} Batch;

static void* worker(void* arg) {
  Batch* b = (Batch*)arg;
  OSolver* s = solver_new(b->tt_log2);
  for (;;) {
    pthread_mutex_lock(&b->mu);
    long job = b->next++;
    pthread_mutex_unlock(&b->mu);
    if (job >= b->n * b->jpd) break;
    long deal = job / b->jpd;
    int sub = (int)(job % b->jpd);
    int strain = b->jpd == 5 ? sub : sub / 4;
    int d0 = b->jpd == 5 ? 0 : sub % 4, d1 = b->jpd == 5 ? 3 : d0;
    u64 before = s->c.nodes;
    solve_job(&s->c, b->hands + deal * 4, strain, d0, d1, b->seeds ? b->seeds + deal * 20 + strain * 4 : NULL,
              b->out20 + deal * 20 + strain * 4);
    if (b->job_nodes) b->job_nodes[job] = s->c.nodes - before;
  }
  pthread_mutex_lock(&b->mu);
  b->nodes += s->c.nodes;
  pthread_mutex_unlock(&b->mu);
  solver_free(s);
  return NULL;
}

/* n deals, all strains and declarers. jpd 5: one job per (deal, strain), the four leads
 * share a TT; 20: one job per (deal, strain, declarer), each from target 7. seeds20: NS
 * seeds (stepping search) or NULL. Returns total nodes, or -1 on bad arguments. */
long long ddo_solve_batch(const uint64_t* hands, long n, int tt_log2, int threads, int jpd,
                          const int8_t* seeds20, int* out20, uint64_t* job_nodes) {
  if (n < 0 || tt_log2 < 9 || tt_log2 > 24 || (jpd != 5 && jpd != 20)) return -1;
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  Batch b;
  b.hands = hands;
  b.n = n;
  b.tt_log2 = tt_log2;
  b.jpd = jpd;
  b.seeds = seeds20;
  b.out20 = out20;
  b.job_nodes = job_nodes;
  b.next = 0;
  b.nodes = 0;
  pthread_mutex_init(&b.mu, NULL);
  pthread_t th[256];
  for (int i = 0; i < threads; i++) pthread_create(&th[i], NULL, worker, &b);
  for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
  pthread_mutex_destroy(&b.mu);
  return (long long)b.nodes;
}

/* One (deal, strain) job at a time on a caller-held context (one TT), as the reference's
 * dd_solve_strain on a DDCtx (src/dd.h:926-939): returns the job's nodes. */
void* ddo_ctx_new(int tt_log2) {
  if (tt_log2 < 9 || tt_log2 > 24) return NULL;
  return solver_new(tt_log2);
}
long long ddo_ctx_solve_strain(void* ctx, const uint64_t* hands4, int strain, int* out4) {
  OSolver* s = (OSolver*)ctx;
  if (!s || strain < 0 || strain > 4) return -1;
  u64 before = s->c.nodes;
  solve_job(&s->c, hands4, strain, 0, 3, NULL, out4);
  return (long long)(s->c.nodes - before);
}
void ddo_ctx_free(void* ctx) {
  if (ctx) solver_free((OSolver*)ctx);
}

/* Unpruned minimax: NS tricks from the position with `leader` to lead (the reference's
 * brute force of tests/test_small.cpp:11-46, for small endings). */
static int brute_rec(OCtx* c) {
  if (c->nplayed == 0 && c->left == 0) return 0;
  int seat = (c->leader + c->nplayed) & 3;
  u64 legal = c->hand[seat];
  if (c->nplayed) {
    u64 f = legal & suit_mask(c->trick[0] >> 4);
    if (f) legal = f;
  }
  int ns = is_ns(seat), best = ns ? -1 : 99;
  for (int card = 0; card < 64; card++) {
    if (!(legal >> card & 1)) continue;
    c->hand[seat] ^= bitc(card);
    c->trick[c->nplayed++] = card;
    int v;
    if (c->nplayed == 4) {
      int w = (c->leader + winner_index(c)) & 3, old = c->leader, saved[4];
      for (int k = 0; k < 4; k++) saved[k] = c->trick[k];
      c->leader = w;
      c->nplayed = 0;
      c->left--;
      v = is_ns(w) + brute_rec(c);
      for (int k = 0; k < 4; k++) c->trick[k] = saved[k];
      c->left++;
      c->nplayed = 4;
      c->leader = old;
    } else {
      v = brute_rec(c);
    }
    c->nplayed--;
    c->hand[seat] ^= bitc(card);
    if (ns ? v > best : v < best) best = v;
  }
  return best;
}

int ddo_brute(const uint64_t* hands, int strain, int leader) {
  OCtx c;
  memset(&c, 0, sizeof(c));
  for (int i = 0; i < 4; i++) c.hand[i] = hands[i];
  c.trump = strain == 4 ? -1 : 3 - strain;
  c.leader = leader;
  c.left = popc(hands[0]);
  return brute_rec(&c);
}
