// The exact double-dummy search of one solver lane, as a resumable stage machine.
//
// A search answers "can NS take >= target tricks?" (null window); the trick count of a
// lead comes from a binary search over targets (first 7, then the previous lead's answer)
// or, with a seed, from stepping up or down from it. This is the reference's method
// (src/dd.h:613-939, src/dd_wave.h:1-147). Node counts equal the reference's because the
// order of moves, the bounds that fire and the TT decisions are the same.
//
// What is new is the layout for a GPU lane: the position lives in registers (hands, the
// current trick packed into one word), the frame on top of the stack too (48 bytes,
// written to the lane's stack in HBM only when a child is entered, read back when it
// returns), and the trick-start TT key is recomputed at the store instead of being kept
// per level. One call of lane_step() runs one stage; a warp runs one stage at a time for
// all lanes that are in it.
#pragma once
#include "ddg_order.cuh"
#include "ddg_tt.cuh"

namespace ddg {

struct Pos {
  u64 h[4];
  u32 trick;  // cards of the current trick in play order, a byte each
  int8_t trump, leader, nplayed, ns_won, left;  // small: lanes live in shared memory
};

// One level of the search (48 bytes; 16-byte aligned in the lane's stack).
struct alignas(16) Frame {
  u64 acc;    // relevant cards gathered from the children so far
  u64 tried;  // cards tried at this node
  u64 mv_lo;  // candidate cards 0..7, a byte each
  u64 mv_hi;  // candidates 8..12 (bytes 0..4), count (byte 5), next index (6), cutting card (7)
  u32 undo;   // the trick's cards when this ply completed it
  u32 info;   // result:1 | seat:2 | need:4 | lb:4 | ub:4 | undo leader:2 | -:7 | win card:8
  u64 pad;
};
static_assert(sizeof(Frame) == 48, "frame is three 16-byte words");

DDG_HD int fr_byte(const Frame& f, int k) {
  u64 w = k < 8 ? f.mv_lo : f.mv_hi;
  return (int)((w >> (8 * (k & 7))) & 0xFF);
}
DDG_HD int fr_move(const Frame& f, int k) { return fr_byte(f, k); }
DDG_HD int fr_n(const Frame& f) { return fr_byte(f, 13); }
DDG_HD int fr_i(const Frame& f) { return fr_byte(f, 14); }
DDG_HD int fr_best(const Frame& f) { return (int)(int8_t)(uint8_t)fr_byte(f, 15); }
DDG_HD void fr_set_hi_byte(Frame& f, int k, int v) {
  int sh = 8 * (k - 8);
  f.mv_hi = (f.mv_hi & ~((u64)0xFF << sh)) | ((u64)(v & 0xFF) << sh);
}
DDG_HD void fr_set_i(Frame& f, int i) { fr_set_hi_byte(f, 14, i); }
DDG_HD void fr_set_best(Frame& f, int c) { fr_set_hi_byte(f, 15, c); }
DDG_HD int fr_result(const Frame& f) { return (int)(f.info & 1); }
DDG_HD int fr_seat(const Frame& f) { return (int)((f.info >> 1) & 3); }
DDG_HD int fr_need(const Frame& f) { return (int)((f.info >> 3) & 15); }
DDG_HD int fr_lb(const Frame& f) { return (int)((f.info >> 7) & 15); }
DDG_HD int fr_ub(const Frame& f) { return (int)((f.info >> 11) & 15); }
DDG_HD int fr_undo_leader(const Frame& f) { return (int)((f.info >> 15) & 3); }
DDG_HD int fr_win_card(const Frame& f) { return (int)(int8_t)(uint8_t)(f.info >> 24); }
DDG_HD void fr_set_result(Frame& f, int v) { f.info = (f.info & ~1u) | (u32)(v & 1); }

DDG_HD void frame_load(Frame& f, const Frame* p) {
#ifdef __CUDA_ARCH__
  const ulonglong2* v = reinterpret_cast<const ulonglong2*>(p);
  ulonglong2 a = v[0], b = v[1], c = v[2];
  f.acc = a.x;
  f.tried = a.y;
  f.mv_lo = b.x;
  f.mv_hi = b.y;
  f.undo = (u32)c.x;
  f.info = (u32)(c.x >> 32);
  f.pad = c.y;
#else
  f = *p;
#endif
}
DDG_HD void frame_store(Frame* p, const Frame& f) {
#ifdef __CUDA_ARCH__
  ulonglong2* v = reinterpret_cast<ulonglong2*>(p);
  v[0] = make_ulonglong2(f.acc, f.tried);
  v[1] = make_ulonglong2(f.mv_lo, f.mv_hi);
  v[2] = make_ulonglong2((u64)f.undo | ((u64)f.info << 32), f.pad);
#else
  *p = f;
#endif
}

// Search counters of one lane (per launch).
// ENTER outcome counts (trivial, last trick, TT hit, quick tricks, later tricks, QT 2nd
// hand, expanded) are diagnostics: kept in the bounds-checked build and the host replay
// (DDG_EXIT_COUNTS), left out of the production kernel, whose per-lane counters live in
// shared memory, where every byte taken from the L1 data cache is felt.
#ifdef DDG_BOUNDS_CHECK
#define DDG_EXIT_COUNTS 1
#endif
struct LaneStats {
  u64 nodes;
  TTStats tt;
#ifdef DDG_EXIT_COUNTS
  u32 enter_exit[7];
#endif
  u32 bounds;         // bounds-checked builds: accesses out of range, skipped
};
#ifdef DDG_EXIT_COUNTS
#define DDG_EXIT(st, k) ((st).enter_exit[k]++)
#else
#define DDG_EXIT(st, k) ((void)0)
#endif

// Frames per lane: the root and at most 52 plies below it, plus one spare (the reference's
// dd_search keeps 53 frames, src/dd.h:802).
#ifndef DDG_STACK_DEPTH
#define DDG_STACK_DEPTH 54
#endif
enum { STACK_DEPTH = DDG_STACK_DEPTH };

// Bounds-checked builds (-DDDG_BOUNDS_CHECK, libddg_check.so): every frame-stack index,
// TT bucket index and task index is checked before its access; a check that fails counts
// in LaneStats::bounds, the access is skipped and the lane stops (its results stay
// unsolved, and the call reports the count as an error). It never traps: the device and
// the context stay usable. In the default build the checks compile to nothing.
#ifdef DDG_BOUNDS_CHECK
#define DDG_IN_BOUNDS(cond, st) ((cond) || ((st).bounds++, false))
#else
#define DDG_IN_BOUNDS(cond, st) true
#endif

DDG_HD int trick_at(const Pos& p, int i) { return trick_card(p.trick, i); }

// Trick winner's index among the first n cards.
DDG_HD int winning_index(const Pos& p, int n) {
  int w = 0;
  for (int i = 1; i < n; i++)
    if (beats(trick_at(p, i), trick_at(p, w), p.trump)) w = i;
  return w;
}

// Candidates of the hand to play: legal cards, one per run of alike cards (`all` gets
// the cards still in play, those of the current trick included).
DDG_HD u64 candidates(const Pos& p, int seat, u64& all) {
  const u64 own = hand_at(p.h, seat);
  u64 legal = own;
  all = all_cards(p.h);
  if (p.nplayed) {
    u64 follow = own & suit_cards(card_suit(trick_at(p, 0)));
    if (follow) legal = follow;
    for (int i = 0; i < p.nplayed; i++) all |= card_bit(trick_at(p, i));
  }
  return legal & run_tops(own, all);
}

// Inserts `card` behind the candidates scoring at least `sc` (ties keep the order of
// arrival, highest card index first), then packs the list into the frame.
DDG_HD void insert_move(int* score, int* card_of, int& n, int card, int sc) {
  int i = n++;
  while (i > 0 && score[i - 1] < sc) {
    score[i] = score[i - 1];
    card_of[i] = card_of[i - 1];
    i--;
  }
  score[i] = sc;
  card_of[i] = card;
}
DDG_HD void pack_moves(Frame& f, const int* card_of, int n) {
  u64 lo = 0, hi = 0;
  for (int k = 0; k < n; k++) {
    if (k < 8) lo |= (u64)card_of[k] << (8 * k);
    else hi |= (u64)card_of[k] << (8 * (k - 8));
  }
  f.mv_lo = lo;
  f.mv_hi = hi | (u64)n << 40 | (u64)0xFF << 56;  // next index 0, no cutting card yet
}

// The leader's candidates at a trick start, best first by the DDS lead weights; `hint`
// (the TT's best move, or -1) and the cards alike to it get the weights' TT bonus.
DDG_CALL void gen_moves_lead(const Pos& p, int hint, Top top, Frame& f) {
  Hands hs;
  for (int i = 0; i < 4; i++) hs.h[i] = p.h[i];
  const int seat = p.leader;
  const u64 own = hand_at(p.h, seat);
  u64 all;
  u64 rest = candidates(p, seat, all);
  int n = 0, score[13], card_of[13];
  while (rest) {
    int card = top_bit(rest);
    rest ^= card_bit(card);
    bool hinted = hint >= 0 && alike(own, all, hint, card);
    insert_move(score, card_of, n, card, lead_weight(hs, top, p.trump, p.left, seat, card, hinted));
  }
  pack_moves(f, card_of, n);
}

// The candidates of the 2nd, 3rd or 4th hand, best first by the DDS follow weights. (The
// reference's TT hint never reaches these: probes happen at trick starts only.)
DDG_CALL void gen_moves_follow(const Pos& p, Frame& f) {
  Hands hs;
  for (int i = 0; i < 4; i++) hs.h[i] = p.h[i];
  const int seat = (p.leader + p.nplayed) & 3;
  u64 all;
  u64 rest = candidates(p, seat, all);
  const Follow fo = follow_init(p.h, p.trump, p.leader, p.trick, p.nplayed);
  int n = 0, score[13], card_of[13];
  while (rest) {
    int card = top_bit(rest);
    rest ^= card_bit(card);
    insert_move(score, card_of, n, card, follow_weight(fo, hs, p.trump, p.nplayed, seat, card));
  }
  pack_moves(f, card_of, n);
}

// Frame of a node that expands: no relevant cards or tried cards yet; `result` starts as
// the value when no child cuts (NS to play fails, EW to play holds). The TT hint waits in
// the frame's spare word until the moves are generated.
DDG_HD void open_frame(Frame& f, int seat, int need, int ub, int hint) {
  f.acc = 0;
  f.tried = 0;
  f.undo = 0;
  f.pad = (u64)(uint8_t)(int8_t)hint;
  f.info = (u32)(!ns_side(seat)) | (u32)seat << 1 | (u32)need << 3 | (u32)ub << 11 | 0xFFu << 24;
}
DDG_HD int frame_hint(const Frame& f) { return (int)(int8_t)(uint8_t)(f.pad & 0xFF); }
// The spare word also records a donation: bits 32..47 = task id + 1 (0 = none), bits
// 48..55 = the frame's candidate count before its tail was donated.
DDG_HD int fr_task(const Frame& f) { return (int)((f.pad >> 32) & 0xFFFF) - 1; }
DDG_HD int fr_full_n(const Frame& f) { return (int)((f.pad >> 48) & 0xFF); }
DDG_HD void fr_set_n(Frame& f, int n) { fr_set_hi_byte(f, 13, n); }
DDG_HD void fr_set_task(Frame& f, int task, int full_n) {
  f.pad = (f.pad & 0xFFFFFFFFull) | ((u64)(task + 1) << 32) | ((u64)full_n << 48);
}
DDG_HD void fr_clear_task(Frame& f) { f.pad &= 0xFFFFFFFFull; }

// ENTER at a trick start (src/dd.h:626-705): cutoffs, the last trick, the TT probe,
// QuickTricks and LaterTricks (their results are stored). Returns 0/1 when decided (`rel`
// set), else -1: the node expands, `top` and the frame are ready for gen_moves_lead.
DDG_CALL int enter_lead(Pos& p, int target, Frame& f, u64& rel, Top& top, TTBucket* tt, u32 mask, u32 gen,
                        LaneStats& st) {
  st.nodes++;
  rel = 0;
  if (p.ns_won >= target) {
    DDG_EXIT(st, 0);
    return 1;
  }
  if (p.ns_won + p.left < target) {
    DDG_EXIT(st, 0);
    return 0;
  }
  const int need = target - p.ns_won;
  const u64 all = all_cards(p.h);
  if (p.left == 1) {
    // Last trick: the highest trump, else the highest card of the suit led.
    int s = (p.trump >= 0 && (all & suit_cards(p.trump))) ? p.trump : card_suit(top_bit(hand_at(p.h, p.leader)));
    u64 in = all & suit_cards(s);
    int hi = top_bit(in);
    if (popc(in) >= 2) rel = card_bit(hi);
    DDG_EXIT(st, 1);
    return ns_side(holder_of(p.h, hi)) ? 1 : 0;
  }
  Hands hs;
  for (int i = 0; i < 4; i++) hs.h[i] = p.h[i];
  const NodeKey key = make_key(hs, p.leader, p.left, gen, mask);
  if (!DDG_IN_BOUNDS(key.bucket <= mask, st)) return 0;
  const ProbeOut pr = tt_probe(tt, key, need, st.tt);
  if (pr.hit >= 0) {
    rel = pr.rel;
    DDG_EXIT(st, 2);
    return pr.hit;
  }
  top = make_top(hs, key.lens);
  const bool ns_lead = ns_side(p.leader);
  const int cut_ns = need, cut_ew = p.left - need + 1;
  const QtOut qo = quick_tricks(hs, top, p.trump, p.leader, ns_lead ? cut_ns : cut_ew, ns_lead ? cut_ew : cut_ns);
  int val = -1;
  u64 wr = 0;
  if (qo.decided) {
    val = ns_lead ? qo.q != 0 : qo.q == 0;
    wr = qo.wr;
    DDG_EXIT(st, 3);
  } else {
    const BoundOut lt = later_tricks(top, p.trump, p.leader, p.ns_won, p.left, target);
    if (lt.v) {
      val = !ns_lead;
      wr = lt.wr;
      DDG_EXIT(st, 4);
    }
  }
  if (val >= 0) {  // one store for both bounds, so lanes that decided either way store together
    tt_store(tt, key, gen, wr, val ? need : 0, val ? p.left : need - 1, -1, st.tt);
    rel = wr;
    return val;
  }
  open_frame(f, p.leader, need, p.left, pr.hint);
  DDG_EXIT(st, 6);
  return -1;
}

// ENTER inside a trick (src/dd.h:706-736): the second hand's QuickTricks. Returns 0/1 when
// decided (`rel` set), else -1: the frame is ready for gen_moves_follow.
DDG_CALL int enter_follow(Pos& p, int target, Frame& f, u64& rel, LaneStats& st) {
  st.nodes++;
  if (p.nplayed == 1) {
    // The trick-start table, with the led card given back to the leader.
    Hands hs, th;
    for (int i = 0; i < 4; i++) hs.h[i] = th.h[i] = p.h[i];
    toggle_card(th.h, p.leader, trick_at(p, 0));
    const Top top = make_top(th, length_key(th.h));
    const int second = lho_of(p.leader);
    const int need2 = target - p.ns_won;
    const int cutoff = ns_side(second) ? need2 : p.left - need2 + 1;
    const BoundOut q2 = quick_tricks_2nd(hs, top, p.trump, second, trick_at(p, 0), cutoff);
    if (q2.v) {
      rel = q2.wr;
      DDG_EXIT(st, 5);
      return ns_side(second) ? 1 : 0;
    }
  }
  open_frame(f, (p.leader + p.nplayed) & 3, 0, 0, -1);
  DDG_EXIT(st, 6);
  return -1;
}

// Plays the frame's card (src/dd.h:739-756); at the fourth card the trick is settled and
// the frame keeps what unplay needs.
DDG_HD void play(Pos& p, Frame& f, int card) {
  const int seat = fr_seat(f);
  toggle_card(p.h, seat, card);
  p.trick = (p.trick & ~(0xFFu << (8 * p.nplayed))) | ((u32)card << (8 * p.nplayed));
  p.nplayed++;
  if (p.nplayed == 4) {
    int wi = winning_index(p, 4);
    int w = (p.leader + wi) & 3;
    int wc = trick_at(p, wi), same = 0;
    for (int k = 0; k < 4; k++) same += card_suit(trick_at(p, k)) == card_suit(wc);
    f.undo = p.trick;
    f.info = (f.info & ~(3u << 15) & ~(0xFFu << 24)) | ((u32)p.leader << 15) |
             ((u32)(same >= 2 ? wc : 0xFF) << 24);  // won by rank: the card is relevant
    p.leader = w;
    p.nplayed = 0;
    p.left--;
    p.ns_won += ns_side(w);
  }
}

DDG_HD void unplay(Pos& p, const Frame& f, int card, u64& rel) {
  if (p.nplayed == 0) {  // this ply completed a trick
    p.trick = f.undo;
    p.ns_won -= ns_side(p.leader);
    p.left++;
    p.nplayed = 4;
    p.leader = fr_undo_leader(f);
    int wc = fr_win_card(f);
    if (wc >= 0) rel |= card_bit(wc);
  }
  p.nplayed--;
  toggle_card(p.h, fr_seat(f), card);
}

// All moves of `f` are done (src/dd.h:772-797): widen the relevant cards through runs of
// the hand's own touching cards, and store trick-start results in the TT.
DDG_CALL u64 finish(const Pos& p, const Frame& f, TTBucket* tt, u32 mask, u32 gen, LaneStats& st) {
  u64 acc = f.acc;
  const u64 own = hand_at(p.h, fr_seat(f));
  u64 all = all_cards(p.h);
  for (int i = 0; i < p.nplayed; i++) all |= card_bit(trick_at(p, i));
  for (int s = 0; s < 4; s++) {
    u64 r = acc & suit_cards(s);
    if (!r) continue;
    int low = low_bit(r);
    while ((own >> low) & 1) {
      u64 below = all & suit_cards(s) & (card_bit(low) - 1);
      if (!below || !((own >> top_bit(below)) & 1)) break;
      low = top_bit(below);
      acc |= card_bit(low);
    }
  }
  if (p.nplayed == 0) {
    int lb = fr_lb(f), ub = fr_ub(f);
    if (fr_result(f)) lb = fr_need(f);
    else ub = fr_need(f) - 1;
    Hands hs;
    for (int i = 0; i < 4; i++) hs.h[i] = p.h[i];
    const NodeKey key = make_key(hs, p.leader, p.left, gen, mask);
    if (DDG_IN_BOUNDS(key.bucket <= mask, st)) tt_store(tt, key, gen, acc, lb, ub, fr_best(f), st.tt);
  }
  return acc;
}

// ---- helping: tasks of donated sibling moves ---------------------------------------------
//
// When the job queue is empty, lanes without work (HUNGRY) help busy lanes, on any SM. A
// lane whose job has run a while donates the untried candidates of its shallowest frame
// whose first child was searched without a cutoff (a node likely to need all its
// children); a helper searches them from that frame's position, with its own TT, and
// reports the value of that part: a cutoff (value, the cutting child's relevant cards and
// card), or no cutoff (the union of the children's relevant cards). The donor merges the
// part into the frame when its own children are done, exactly as if it had searched them
// itself: cutoffs are exact, and a card skipped as a small card is skipped on the evidence
// of a child whose relevant cards are in the frame's set. Node counts then differ from the
// sequential search; tricks do not. A donor never waits on a task nobody has taken (it
// takes the moves back), and waits are checked once per block iteration, never spun on:
// every wait is on a lane that is searching in a resident block, so the launch finishes.
enum { TASK_FREE = 0, TASK_QUEUED = 1, TASK_RUNNING = 2, TASK_DONE = 3, TASK_ABANDONED = 4, TASK_FILLING = 5 };
enum { MAX_TASKS = 1024, CLAIM_WINDOW = 64, MAX_DONATE_DEPTH = 28, DONATE_MIN_NODES = 4096 };

struct Task {
  Pos pos;          // position at the donated frame, before its next candidate
  u64 mv_lo, mv_hi;  // the donated candidates, packed as in a frame (count in byte 13)
  u64 acc, tried;   // the donor frame's relevant and tried cards at the donation
  u64 r;            // result: relevant cards of the donated part
  u32 info;         // the donor frame's info word (seat, result so far)
  int8_t target;    // the null-window target of the donor's search
  int8_t v;         // result: value of the donated part
  int8_t best;      // result: the cutting card, or -1
  u64 key;          // (deal << 3 | strain) + 1 of the donor: helpers keep their TT per key
  int32_t owner;    // the lane whose TT the donor's search uses (shared-TT helping)
  u32 gen;          // that TT's generation for the donor's job
};

// The tasks of a launch and the counters that steer helping (HBM on the GPU).
struct TaskPool {
  Task t[MAX_TASKS];
  int state[MAX_TASKS];
  int queued;     // tasks queued, or reserved by a donor about to post one
  int posted;     // tasks posted so far
  int hungry;     // lanes waiting for a task
  int busy;       // lanes holding a job or a task
  int exhausted;  // the job queue is empty
};

DDG_HD int atom_cas(int* p, int cmp, int val) {
#ifdef __CUDA_ARCH__
  return atomicCAS(p, cmp, val);
#else
  int old = *p;
  if (old == cmp) *p = val;
  return old;
#endif
}
DDG_HD void atom_add(int* p, int v) {
#ifdef __CUDA_ARCH__
  atomicAdd(p, v);
#else
  *p += v;
#endif
}
DDG_HD int atom_load(const int* p) {
#ifdef __CUDA_ARCH__
  return *(const volatile int*)p;
#else
  return *p;
#endif
}
DDG_HD void fence_block() {
#ifdef __CUDA_ARCH__
  __threadfence();  // task records travel between SMs
#endif
}

// Publishes a task (its `queued` slot was reserved by the donor); its id, or -1 when the
// pool is full. The search for a free slot starts at `start` to spread donors out.
DDG_HD int task_post(TaskPool& tp, const Task& t, int start) {
  for (int j = 0; j < MAX_TASKS; j++) {
    const int k = (start + j) & (MAX_TASKS - 1);
    if (atom_load(&tp.state[k]) != TASK_FREE || atom_cas(&tp.state[k], TASK_FREE, TASK_FILLING) != TASK_FREE)
      continue;
    tp.t[k] = t;
    fence_block();
    atom_cas(&tp.state[k], TASK_FILLING, TASK_QUEUED);
    atom_add(&tp.posted, 1);
    return k;
  }
  return -1;
}
// Takes a queued task from a window of the pool starting at `start`; its id, or -1.
DDG_HD int task_claim(TaskPool& tp, int start) {
  if (atom_load(&tp.queued) <= 0) return -1;
  start &= (MAX_TASKS - 1) & ~(CLAIM_WINDOW - 1);  // a window-aligned block of the pool
  u64 queued = 0;  // bit j: slot start + j looked queued
#ifdef __CUDA_ARCH__
  // One pass of vector loads (all in flight at once) from L2, where the atomics live.
  const int4* w = reinterpret_cast<const int4*>(tp.state + start);
#pragma unroll
  for (int j = 0; j < CLAIM_WINDOW / 4; j++) {
    const int4 v = __ldcg(w + j);
    queued |= (u64)(v.x == TASK_QUEUED) << (4 * j) | (u64)(v.y == TASK_QUEUED) << (4 * j + 1) |
              (u64)(v.z == TASK_QUEUED) << (4 * j + 2) | (u64)(v.w == TASK_QUEUED) << (4 * j + 3);
  }
#else
  for (int j = 0; j < CLAIM_WINDOW; j++) queued |= (u64)(tp.state[start + j] == TASK_QUEUED) << j;
#endif
  for (; queued; queued &= queued - 1) {
    const int k = start + low_bit(queued);
    if (atom_cas(&tp.state[k], TASK_QUEUED, TASK_RUNNING) == TASK_QUEUED) {
      atom_add(&tp.queued, -1);
      fence_block();
      return k;
    }
  }
  return -1;
}
// Reads task k written by a lane of another SM, after its state showed it published (a
// claimed task's position) or finished (its result): an acquire fence, then loads from
// L2, since this SM's L1 may still hold the slot's earlier contents.
static_assert(sizeof(Task) % 8 == 0, "task records are read as 8-byte words");
DDG_HD void task_read(const TaskPool& tp, int k, Task& out) {
#ifdef __CUDA_ARCH__
  __threadfence();
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(&tp.t[k]);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&out);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(Task) / 8); i++) d[i] = __ldcg(s + i);
#else
  out = tp.t[k];
#endif
}
// Takes an unclaimed task back; true when it was still queued.
DDG_HD bool task_retract(TaskPool& tp, int k) {
  if (atom_cas(&tp.state[k], TASK_QUEUED, TASK_FREE) == TASK_QUEUED) {
    atom_add(&tp.queued, -1);
    return true;
  }
  return false;
}
// The helper's result; a task abandoned meanwhile is simply freed.
DDG_HD void task_finish(TaskPool& tp, int k, int v, u64 r, int best) {
  tp.t[k].v = (int8_t)v;
  tp.t[k].r = r;
  tp.t[k].best = (int8_t)best;
  fence_block();
  if (atom_cas(&tp.state[k], TASK_RUNNING, TASK_DONE) != TASK_RUNNING) tp.state[k] = TASK_FREE;
}
// The donor no longer needs the task (its own part cut off).
DDG_HD void task_abandon(TaskPool& tp, int k) {
  for (;;) {
    int s = atom_load(&tp.state[k]);
    if (s == TASK_QUEUED) {
      if (task_retract(tp, k)) return;
    } else if (s == TASK_RUNNING) {
      if (atom_cas(&tp.state[k], TASK_RUNNING, TASK_ABANDONED) == TASK_RUNNING) return;
    } else {  // done: free it (abandoned or free already: nothing to do)
      if (s == TASK_DONE) atom_cas(&tp.state[k], TASK_DONE, TASK_FREE);
      return;
    }
  }
}

// ---- the stage machine ------------------------------------------------------------------

enum Stage {
  ST_TAKE = 0,
  ST_ROOT = 1,
  ST_ENTER = 2,
  ST_NEXT = 3,
  ST_RET = 4,
  ST_IDLE = 5,
  ST_MOVES_LEAD = 6,    // the node expands: generate the leader's ordered moves
  ST_MOVES_FOLLOW = 7,  // the node expands: generate a follower's ordered moves
  ST_HUNGRY = 8,        // no job left: waits for a task of its block to help with
  ST_WAIT = 9,          // a frame's own children are done; its donated part is still running
  ST_COUNT = 10
};

// How a lead's trick count is found.
enum { MODE_BISECT = 0, MODE_STEP = 1 };
// Phases of MODE_STEP: first search at the seed, stepping up, stepping down.
enum { PH_FIRST = 0, PH_UP = 1, PH_DOWN = 2 };

// A lane's whole state between stages (192 bytes; in shared memory on the GPU).
struct Lane {
  Pos p;
  Frame f;    // top of the stack
  Frame par;  // copy of the frame last pushed to the stack (depth par_sp): most pops need no load
  Top top;    // trick-start table of an expanding lead node (ENTER -> MOVES_LEAD)
  u64 r;    // relevant cards of the node just finished
  long long job, deal;
  u32 gen;           // generation of the lane's own TT
  int32_t owner;     // shared-TT helping: the lane whose TT this task's search uses, -1 = own
  u32 hgen;          // and that TT's generation for the donor's job
  int16_t task;      // the task this lane helps with, or -1 (its own job)
  int8_t par_sp;     // depth of `par`, or -1
  int8_t stage, sp;  // sp = depth of f; frames 0..sp-1 are in the lane's stack
  int8_t target;     // the null-window search in progress: NS >= target?
  int8_t lo, hi;     // MODE_BISECT: answer in [lo, hi]; MODE_STEP: lo = t, hi = phase
  int8_t mode, decl, last_decl, strain;
  int8_t v;  // value of the node just finished
};

// The TT a lane's search reads and writes, and its generation: the lane's own, or, for a
// helper with shared-TT helping, the donor's (entries are facts about positions of one
// deal and trump, so every lane searching parts of one job may share them; a helper's
// findings then serve the donor and the other helpers of the job, and theirs serve it).
template <class Env>
DDG_HD TTBucket* search_tt(const Lane& L, Env& env) {
  return L.owner >= 0 ? env.tt_of(L.owner) : env.tt;
}
DDG_HD u32 search_gen(const Lane& L) { return L.owner >= 0 ? L.hgen : L.gen; }

// Sets up the search of declarer `decl`'s lead (leader = decl + 1) at `target`.
DDG_HD void start_search(Lane& L) {
  fr_set_best(L.f, -1);  // no root card yet (a root decided without moves keeps none)
  L.p.leader = (L.decl + 1) & 3;
  L.p.nplayed = 0;
  L.p.ns_won = 0;
  L.p.left = popc(L.p.h[0]);
  L.p.trick = 0;
  L.sp = 0;
  L.par_sp = -1;
  L.stage = ST_ENTER;
}

// Starts the trick count of the current declarer: the binary search at `first`, or the
// stepping search from the seed `first`.
DDG_HD void start_lead(Lane& L, int first) {
  if (L.mode == MODE_BISECT) {
    L.lo = 0;
    L.hi = 13;
    L.target = first < 1 ? 1 : first > 13 ? 13 : first;
    start_search(L);
    return;
  }
  int left = popc(L.p.h[0]);
  int t = first < 0 ? 0 : first > left ? left : first;
  L.lo = t;
  if (t == 0) {  // ">= 0" needs no search
    L.hi = PH_UP;
    L.target = 1;
  } else {
    L.hi = PH_FIRST;
    L.target = t;
  }
  if (L.hi == PH_UP && L.lo >= left) {
    L.target = -1;  // answer known: lo
    return;
  }
  start_search(L);
}

// A root search finished with L.v: next target, or the lead's answer (>= 0) when known.
DDG_HD int root_result(Lane& L) {
  if (L.mode == MODE_BISECT) {
    if (L.v) L.lo = L.target;
    else L.hi = L.target - 1;
    if (L.lo < L.hi) {
      L.target = (L.lo + L.hi + 1) / 2;
      return -1;
    }
    return L.lo;
  }
  int left = popc(L.p.h[0]);
  int t = L.lo;
  if (L.hi == PH_FIRST || L.hi == PH_UP) {
    if (L.hi == PH_FIRST && !L.v) {
      t--;
      L.lo = t;
      L.hi = PH_DOWN;
      if (t <= 0) return 0;
      L.target = t;
      return -1;
    }
    if (L.hi == PH_UP) {
      if (!L.v) return t;
      t++;
    }
    L.lo = t;
    L.hi = PH_UP;
    if (t >= left) return t;
    L.target = t + 1;
    return -1;
  }
  // PH_DOWN: searching t
  if (L.v) return t;
  t--;
  L.lo = t;
  if (t <= 0) return 0;
  L.target = t;
  return -1;
}

// The environment a lane runs in (a GPU block, or the host replay in the tests):
//   bool take(Lane&)            next job: fills deal, strain, decl, last_decl, mode, hands;
//                               false when there is none
//   int seed(const Lane&)       first target / seed of the current declarer
//   void answer(const Lane&, int tricks)  result of the current declarer
//   void job_done(const Lane&)  the lane's job is finished
//   Frame* stack                the lane's frames (depth 0..52)
//   TTBucket* tt; u32 mask      the lane's TT
//   LaneStats& stats()          the lane's counters (kept out of registers on the GPU)
template <class Env>
DDG_CALL void node_done(Lane& L, Env& env) {
  if (L.sp > 0) {
    if (!DDG_IN_BOUNDS(L.sp <= STACK_DEPTH, env.stats())) {
      L.stage = ST_IDLE;
      return;
    }
    L.sp--;
    if (L.par_sp == L.sp) L.f = L.par;  // the frame pushed last: still in shared memory
    else frame_load(L.f, env.stack + L.sp);
    L.par_sp = -1;
    if (L.sp > 0) {  // the next pop's frame, on its way to L1
      const char* g = reinterpret_cast<const char*>(env.stack + L.sp - 1);
      prefetch_l1(g);
      prefetch_l1(g + sizeof(Frame) - 1);
    }
    L.stage = ST_RET;
    return;
  }
  // A root search that went the leader's way names the lead that did it (the cutting
  // card): after the last such search it is a best lead for the answer.
  if (L.task < 0 && (L.v != 0) == ((L.p.leader & 1) == 0)) {
    const int b = fr_best(L.f);
    if (b >= 0) env.root_best(L, b);
  }
  int ans = root_result(L);
  if (ans < 0) {
    start_search(L);
    return;
  }
  for (;;) {
    env.answer(L, ans);
    L.decl++;
    if (L.decl > L.last_decl) {
      env.job_done(L);
      if (env.pool()) atom_add(&env.pool()->busy, -1);
      L.stage = ST_TAKE;
      return;
    }
    // The next lead starts at this answer (binary search) or at its own seed.
    start_lead(L, L.mode == MODE_BISECT ? ans : env.seed(L));
    if (L.target >= 0) return;
    ans = L.lo;
  }
}

// ---- one stage of one lane -------------------------------------------------------------
//
// Besides the members listed above node_done, an Env offers helping:
//   TaskPool* pool()        the launch's tasks and helping counters, or null (helping off)
//   bool want_donation()    a hungry lane has no task waiting for it: reserves one
//   void unreserve()        gives back a reservation that was not used
//   int claim_start()       where this lane starts looking for a task in the pool
//   u64 work_nodes()        nodes searched since the lane's job or task began

template <class Env>
DDG_CALL void step_take(Lane& L, Env& env) {
  TaskPool* tp = env.pool();
  // Shared-TT helping: helpers still writing into this lane's TT (an abandoned task that
  // has not yet seen it is abandoned) hold the TT for the finished job; the next job, with
  // its new generation and possibly a tag clear, waits for them.
  if (tp && env.share_tt() && env.tt_users(env.self()) > 0) {
    L.stage = ST_TAKE;
    return;
  }
  const int got = env.take(L);
  if (got < 0) {  // a stream with no deal published yet: try again later
    L.stage = ST_TAKE;
    return;
  }
  if (!got) {
    if (tp) {
      tp->exhausted = 1;
      atom_add(&tp->hungry, 1);
      L.stage = ST_HUNGRY;
    } else {
      L.stage = ST_IDLE;
    }
    return;
  }
  if (tp) atom_add(&tp->busy, 1);
  L.task = -1;
  L.owner = -1;
  L.p.trump = strain_trump(L.strain);
  L.p.trick = 0;
  L.gen = tt_next_gen(env.tt, env.mask, L.gen);
  env.tt_key() = 0;
  L.stage = ST_ROOT;
}

template <class Env>
DDG_CALL void step_root(Lane& L, Env& env) {
  start_lead(L, env.seed(L));
  if (L.target >= 0) return;
  // Answered without a search (a seed of 0 with no tricks left).
  L.sp = 0;
  L.par_sp = -1;
  L.v = 1;
  int ans = L.lo;
  for (;;) {
    env.answer(L, ans);
    L.decl++;
    if (L.decl > L.last_decl) {
      env.job_done(L);
      if (env.pool()) atom_add(&env.pool()->busy, -1);
      L.stage = ST_TAKE;
      return;
    }
    start_lead(L, L.mode == MODE_BISECT ? ans : env.seed(L));
    if (L.target >= 0) return;
    ans = L.lo;
  }
}

// ENTER: decided at once (node done), or the node expands (moves next).
template <class Env>
DDG_HD void step_enter(Lane& L, Env& env) {
  const bool lead = L.p.nplayed == 0;
  int e = lead ? enter_lead(L.p, L.target, L.f, L.r, L.top, search_tt(L, env), env.mask, search_gen(L),
                            env.stats())
               : enter_follow(L.p, L.target, L.f, L.r, env.stats());
  if (e < 0) {
    L.stage = lead ? ST_MOVES_LEAD : ST_MOVES_FOLLOW;
    return;
  }
  L.v = e;
  node_done(L, env);
}

template <class Env>
DDG_CALL void step_moves(Lane& L, Env& env) {
  if (L.stage == ST_MOVES_LEAD) {
    int hint = frame_hint(L.f);
    // At a job's root with no TT move yet, an outside hint (the learned guide's lead) takes
    // the TT move's place in the ordering; the searches still decide every answer.
    if (hint < 0 && L.sp == 0 && L.task < 0) {
      const int h = env.root_hint(L);
      if (h >= 0 && h < 64 && (hand_at(L.p.h, L.p.leader) >> h & 1)) hint = h;
    }
    gen_moves_lead(L.p, hint, L.top, L.f);
  } else {
    gen_moves_follow(L.p, L.f);
  }
  L.stage = ST_NEXT;
}

// The top frame is done with value L.v: a helper's task root reports to its donor (no
// widening, no TT store: the frame holds only part of the node's moves); any other
// frame is finished and returns to its parent.
template <class Env>
DDG_CALL void frame_done(Lane& L, Env& env) {
  Frame& f = L.f;
  if (L.sp == 0 && L.task >= 0) {
    if (!DDG_IN_BOUNDS(L.task < MAX_TASKS, env.stats())) {
      L.stage = ST_IDLE;
      return;
    }
    TaskPool& tp = *env.pool();
    task_finish(tp, L.task, L.v, f.acc, fr_best(f));
    L.task = -1;
    if (L.owner >= 0) {  // done with the donor's TT
      env.tt_users_add(L.owner, -1);
      L.owner = -1;
    }
    atom_add(&tp.busy, -1);
    atom_add(&tp.hungry, 1);
    L.stage = ST_HUNGRY;
    return;
  }
  L.r = finish(L.p, f, search_tt(L, env), env.mask, search_gen(L), env.stats());
  node_done(L, env);
}

// NEXT: play the frame's next candidate (src/dd.h:812-835), or finish the node.
template <class Env>
DDG_CALL void step_next(Lane& L, Env& env) {
  Frame& f = L.f;
  for (;;) {
    int i = fr_i(f);
    const int n = fr_n(f);
    if (!DDG_IN_BOUNDS(n <= 13 && L.sp < STACK_DEPTH, env.stats())) {
      L.stage = ST_IDLE;
      return;
    }
    while (i < n) {
      int card = fr_move(f, i);
      int s = card_suit(card);
      // Cards below every relevant card of their suit are alike: one of them is tried.
      u64 rs = f.acc & suit_cards(s);
      u64 small = rs ? (card_bit(low_bit(rs)) - 1) & suit_cards(s) : suit_cards(s);
      if ((small & card_bit(card)) && (small & f.tried)) {
        i++;
        continue;
      }
      fr_set_i(f, i);
      f.tried |= card_bit(card);
      play(L.p, f, card);
      frame_store(env.stack + L.sp, f);
      L.par = f;
      L.par_sp = L.sp;
      L.sp++;
      if (L.p.nplayed == 0)  // a trick start next: its TT tag line, on its way to L2
        prefetch_l2(search_tt(L, env) + (key_hash(length_key(L.p.h), L.p.leader) & env.mask));
      L.stage = ST_ENTER;
      return;
    }
    fr_set_i(f, i);
    const int t = fr_task(f);
    if (t < 0) break;
    if (!DDG_IN_BOUNDS(t < MAX_TASKS, env.stats())) {
      L.stage = ST_IDLE;
      return;
    }
    // Own children done; the donated tail decides what comes next.
    TaskPool& tp = *env.pool();
    if (task_retract(tp, t)) {  // nobody took it: search it here after all
      fr_set_n(f, fr_full_n(f));
      fr_clear_task(f);
      continue;
    }
    if (atom_load(&tp.state[t]) != TASK_DONE) {
      L.stage = ST_WAIT;
      return;
    }
    Task k;
    task_read(tp, t, k);
    if (k.v == (int)ns_side(fr_seat(f))) {  // the donated part cut off
      fr_set_result(f, k.v);
      f.acc = k.r;
      fr_set_best(f, k.best);
    } else {
      f.acc |= k.r;
    }
    fence_block();  // the result is read before the slot can be posted again
    tp.state[t] = TASK_FREE;
    fr_clear_task(f);
    break;
  }
  L.v = fr_result(f);
  frame_done(L, env);
}

// RET: the child of the top frame returned (L.v, L.r) (src/dd.h:840-854).
template <class Env>
DDG_CALL void step_ret(Lane& L, Env& env) {
  Frame& f = L.f;
  int card = fr_move(f, fr_i(f));
  unplay(L.p, f, card, L.r);
  if (L.v == (int)ns_side(fr_seat(f))) {  // the child cuts
    const int t = fr_task(f);
    if (t >= 0 && DDG_IN_BOUNDS(t < MAX_TASKS, env.stats())) {  // the donated tail is not needed any more
      task_abandon(*env.pool(), t);
      fr_clear_task(f);
    }
    fr_set_result(f, L.v);
    f.acc = L.r;
    fr_set_best(f, card);
    frame_done(L, env);
    return;
  }
  f.acc |= L.r;
  fr_set_i(f, fr_i(f) + 1);
  L.stage = ST_NEXT;
}

// WAIT: the top frame's donated tail is running on a helper.
template <class Env>
DDG_HD bool step_wait(Lane& L, Env& env) {
  if (!DDG_IN_BOUNDS(fr_task(L.f) >= 0 && fr_task(L.f) < MAX_TASKS, env.stats())) {
    L.stage = ST_IDLE;
    return false;
  }
  if (atom_load(&env.pool()->state[fr_task(L.f)]) != TASK_DONE) return false;
  L.stage = ST_NEXT;  // NEXT merges the result and finishes the frame
  return true;
}

// HUNGRY: take a task of the block, or stop when nothing is left to do.
template <class Env>
DDG_CALL bool step_hungry(Lane& L, Env& env) {
  TaskPool& tp = *env.pool();
  const int t = task_claim(tp, env.claim_start());
  if (t < 0) {
    if (atom_load(&tp.exhausted) && atom_load(&tp.busy) == 0) {  // nothing left anywhere
      atom_add(&tp.hungry, -1);
      L.stage = ST_IDLE;
    }
    return false;
  }
  atom_add(&tp.hungry, -1);
  atom_add(&tp.busy, 1);
  env.task_started();
  Task k;
  task_read(tp, t, k);
  L.p = k.pos;
  L.f.acc = k.acc;
  L.f.tried = k.tried;
  L.f.mv_lo = k.mv_lo;
  L.f.mv_hi = k.mv_hi;
  L.f.undo = 0;
  L.f.info = k.info;
  L.f.pad = 0;
  L.sp = 0;
  L.par_sp = -1;
  L.target = k.target;
  L.task = (int16_t)t;
  L.deal = (long long)((k.key - 1) >> 3);
  L.strain = (int8_t)((k.key - 1) & 7);
  L.stage = ST_NEXT;
  if (env.share_tt()) {
    // The helper searches in the donor's TT. It registers as a user of that TT first and
    // then checks that the task is still running: a donor abandons a task before it can
    // finish its job, and looks at its TT's users only after that, so either it sees this
    // helper registered, or the helper sees the task abandoned and stops before touching
    // the TT.
    env.tt_users_add(k.owner, 1);
    L.owner = k.owner;
    L.hgen = k.gen;
    fence_block();
    if (atom_load(&tp.state[t]) == TASK_ABANDONED) abort_task(L, env);
    return true;
  }
  // Entries of the TT are facts about positions of one deal and trump suit: a helper that
  // stays on the same (deal, strain) keeps them, which spares it re-searching the subtrees
  // its earlier tasks already solved.
  if (env.tt_key() != k.key) {
    L.gen = tt_next_gen(env.tt, env.mask, L.gen);
    env.tt_key() = k.key;
  }
  return true;
}

// A helper whose task was abandoned stops, and abandons what it had donated itself.
template <class Env>
DDG_CALL void abort_task(Lane& L, Env& env) {
  TaskPool& tp = *env.pool();
  if (!DDG_IN_BOUNDS(L.sp <= STACK_DEPTH && L.task >= 0 && L.task < MAX_TASKS, env.stats())) {
    L.stage = ST_IDLE;
    return;
  }
  for (int k = 0; k < L.sp; k++) {
    Frame g;
    frame_load(g, env.stack + k);
    if (fr_task(g) >= 0 && DDG_IN_BOUNDS(fr_task(g) < MAX_TASKS, env.stats())) task_abandon(tp, fr_task(g));
  }
  // In NEXT, RET and WAIT the top frame is the one at depth sp; in ENTER and MOVES it is
  // the copy of frame sp-1 (done above) or a fresh frame without a task.
  const bool top_is_own = L.stage == ST_NEXT || L.stage == ST_RET || L.stage == ST_WAIT;
  if (top_is_own && fr_task(L.f) >= 0 && DDG_IN_BOUNDS(fr_task(L.f) < MAX_TASKS, env.stats()))
    task_abandon(tp, fr_task(L.f));
  if (L.owner >= 0) {  // no more writes into the donor's TT
    fence_block();
    env.tt_users_add(L.owner, -1);
    L.owner = -1;
  }
  tp.state[L.task] = TASK_FREE;
  L.task = -1;
  atom_add(&tp.busy, -1);
  atom_add(&tp.hungry, 1);
  L.stage = ST_HUNGRY;
}
DDG_HD bool task_abandoned(const Lane& L, const TaskPool* tp) {
  return L.task >= 0 && atom_load(&tp->state[L.task]) == TASK_ABANDONED;
}

// Donates the untried tail of the shallowest frame (below the top) whose first child was
// searched without a cutoff. The lane is in NEXT, so its position is that of the top
// frame; the donated frame's position is found by taking back the moves above it.
template <class Env>
DDG_CALL bool try_donate(Lane& L, Env& env) {
  if (!DDG_IN_BOUNDS(L.sp <= STACK_DEPTH, env.stats())) return false;
  const int top = L.sp < MAX_DONATE_DEPTH ? L.sp : MAX_DONATE_DEPTH;
  for (int d = 0; d < top; d++) prefetch_l1(env.stack + d);  // the scan's loads, in flight together
  for (int d = 0; d < top; d++) {
    Frame g;
    frame_load(g, env.stack + d);
    const int i = fr_i(g), n = fr_n(g);
    if (fr_task(g) >= 0 || i < 1 || n - i < 2) continue;
    Task t;
    t.pos = L.p;
    for (int j = L.sp - 1; j >= d; j--) {
      Frame h;
      if (j == d) h = g;
      else frame_load(h, env.stack + j);
      u64 dummy = 0;
      unplay(t.pos, h, fr_move(h, fr_i(h)), dummy);
    }
    int cards[13], m = 0;
    for (int k = i + 1; k < n; k++) cards[m++] = fr_move(g, k);
    Frame tail;
    pack_moves(tail, cards, m);
    t.mv_lo = tail.mv_lo;
    t.mv_hi = tail.mv_hi;
    // The child the donor is still searching counts as not tried for the helper: its
    // relevant cards are not in acc yet, so it cannot justify skipping a small card.
    t.acc = g.acc;
    t.tried = g.tried & ~card_bit(fr_move(g, i));
    t.info = g.info;
    t.target = L.target;
    t.key = ((u64)L.deal << 3 | (u64)L.strain) + 1;
    t.owner = L.owner >= 0 ? L.owner : (int32_t)env.self();  // a helper passes its donor's TT on
    t.gen = search_gen(L);
    t.r = 0;
    t.v = 0;
    t.best = -1;
    const int id = task_post(*env.pool(), t, env.claim_start());
    if (id < 0) return false;
    fr_set_task(g, id, n);
    fr_set_n(g, i + 1);
    frame_store(env.stack + d, g);
    if (L.par_sp == d) L.par = g;
    return true;
  }
  return false;
}

DDG_HD bool cheap_stage(int st) {
  return st == ST_RET || st == ST_NEXT || st == ST_ROOT || st == ST_TAKE || st == ST_HUNGRY || st == ST_WAIT;
}

// Runs the cheap stages back to back until the lane needs ENTER, waits, or has nothing
// left. A lane about to play its next move first donates when its block is hungry.
template <class Env>
DDG_CALL void advance_cheap(Lane& L, Env& env) {
  bool offered = false;
  const int limit = env.cheap_limit();
  for (int k = 1;; k++) {
    if (limit && k > limit) return;  // the rest waits for the next pass
    switch (L.stage) {
      case ST_RET: step_ret(L, env); break;
      case ST_NEXT:
        if (!offered && env.pool() && L.sp > 0 && env.work_nodes() >= DONATE_MIN_NODES && env.want_donation()) {
          offered = true;
          if (!try_donate(L, env)) env.unreserve();
        }
        step_next(L, env);
        break;
      case ST_ROOT: step_root(L, env); break;
      case ST_TAKE:
        step_take(L, env);
        if (L.stage == ST_TAKE) return;  // nothing to take yet
        break;
      case ST_ENTER:  // inside a trick, ENTER is short: run it here when the schedule says so
        if (L.p.nplayed == 0 || !env.fuse_follow()) return;
        step_enter(L, env);
        break;
      case ST_WAIT:
        if (!step_wait(L, env)) return;
        break;
      case ST_HUNGRY:
        if (!step_hungry(L, env)) return;
        break;
      default: return;
    }
  }
}

// Up to `max_steps` stages of one lane, whatever they are: the free-running mode of a block
// with few busy lanes (each thread then runs its own lane without waiting for the others).
// A hungry lane looks for a task only when `may_claim`; a waiting lane stops until its
// helper is done.
template <class Env>
DDG_CALL void advance_free(Lane& L, Env& env, int max_steps, bool may_claim) {
  bool offered = false;
  for (int k = 0; k < max_steps; k++) {
    switch (L.stage) {
      case ST_IDLE: return;
      case ST_HUNGRY:
        if (!may_claim || !step_hungry(L, env)) return;
        may_claim = false;
        break;
      case ST_WAIT:
        if (!step_wait(L, env)) return;
        break;
      case ST_NEXT:
        if (!offered && env.pool() && L.sp > 0 && env.work_nodes() >= DONATE_MIN_NODES && env.want_donation()) {
          offered = true;
          if (!try_donate(L, env)) env.unreserve();
        }
        step_next(L, env);
        break;
      case ST_TAKE:
        step_take(L, env);
        if (L.stage == ST_TAKE) return;
        break;
      case ST_ROOT: step_root(L, env); break;
      case ST_ENTER: step_enter(L, env); break;
      case ST_MOVES_LEAD:
      case ST_MOVES_FOLLOW: step_moves(L, env); break;
      case ST_RET: step_ret(L, env); break;
      default: return;
    }
  }
}

// One stage of the lane, whatever it is (the host replay steps lanes this way).
template <class Env>
DDG_HD void lane_step(Lane& L, Env& env) {
  switch (L.stage) {
    case ST_TAKE: step_take(L, env); return;
    case ST_ROOT: step_root(L, env); return;
    case ST_ENTER: step_enter(L, env); return;
    case ST_MOVES_LEAD:
    case ST_MOVES_FOLLOW: step_moves(L, env); return;
    case ST_NEXT: step_next(L, env); return;
    case ST_RET: step_ret(L, env); return;
    case ST_WAIT: step_wait(L, env); return;
    case ST_HUNGRY: step_hungry(L, env); return;
    default: return;
  }
}

}  // namespace ddg
