// dd_solve.hpp - the reference's header-level solve API, shaped like src/dd.h, over the
// C ABI of libddg.so (include/ddg.h). Code written against hsperr/dds_gpu's
//   DDCtx c{}; c.tt = ...; dd_solve_strain(c, hands, strain, out4);
// compiles against this header with `ddg::DDCtx` (the TT is owned by the context; there
// is no TT pointer to set) and then runs the search on the GPU. Every call is a GPU
// launch; callers with many deals should use dd_solve_deals / ddg_solve_batch.
//
//   reference (src/dd.h)                                 here
//   void dd_solve_strain(DDCtx&, hands, strain, out4)    dd_solve_strain (same arguments)   :926
//   void dd_solve_strain_guess(DDCtx&, hands, strain,    dd_solve_strain_guess              :915
//                              ns4, out4)
//   int dd_ns_tricks(DDCtx&, leader, guess)              dd_ns_tricks (reads c.hand, c.trump) :877
//   int dd_ns_tricks_from(DDCtx&, leader, guess)         dd_ns_tricks_from                  :898
//   void dd_next_gen(DDCtx&)                             dd_next_gen (no effect, see below) :864
//   int dd_strain_suit(int strain)                        dd_strain_suit                     :893
//   uint64_t DDCtx::nodes (accumulates over calls)        DDCtx::nodes                       :119
// Not offered: dd_search (src/dd.h:801), one null-window search from the context's
// current mid-play position (c.leader, c.nplayed, c.ns_won, c.left set by the caller): the
// GPU solves whole leads from the deal, and a single search's relevant-card mask is not
// part of any result the library returns.
// TT generations: every GPU job starts a fresh TT generation, so dd_next_gen has nothing
// left to do; two dd_ns_tricks calls therefore do not share TT entries as they do in the
// reference when the caller skips dd_next_gen between them (same tricks, other node counts).
// Errors: the reference has no error returns; these functions throw ddg::Error with
// ddg_last_error()'s message (bad deal, strain out of range, CUDA failure).
#pragma once
#include <stdint.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "ddg.h"

namespace ddg {

struct Error : std::runtime_error {
  explicit Error(const std::string& m) : std::runtime_error(m) {}
};

inline void check(int rc, const char* what) {
  if (rc != DDG_OK) throw Error(std::string(what) + ": " + ddg_last_error());
}

// Owns one solver pool on a GPU. tt_log2 as the reference's TT_LOG2 (>= 9). `hand` and
// `trump` are the deal and trump suit the one-lead calls read, as the reference's DDCtx
// fields of the same names (src/dd.h:113-125; trump -1 = no trump).
struct DDCtx {
  ddg_solver* solver = nullptr;
  uint64_t nodes = 0;
  uint64_t hand[4] = {0, 0, 0, 0};
  int trump = -1;
  explicit DDCtx(int tt_log2 = 10, int device = 0, int lanes = 0, int jobs_per_deal = 5) {
    ddg_config c;
    ddg_config_default(&c);
    c.tt_log2 = tt_log2;
    c.device = device;
    c.lanes = lanes;
    c.jobs_per_deal = jobs_per_deal;
    check(ddg_solver_create(&c, &solver), "ddg_solver_create");
  }
  ~DDCtx() { ddg_solver_destroy(solver); }
  DDCtx(const DDCtx&) = delete;
  DDCtx& operator=(const DDCtx&) = delete;
};

inline int dd_strain_suit(int strain) { return strain == 4 ? -1 : 3 - strain; }
inline int dd_suit_strain(int trump) { return trump < 0 ? 4 : 3 - trump; }

inline void dd_next_gen(DDCtx&) {}

// Tricks for declarers N,E,S,W in `strain` (E/W: 13 - NS tricks, as the reference).
inline void dd_solve_strain(DDCtx& c, const uint64_t* hands, int strain, int* out4) {
  check(ddg_solve_strain(c.solver, hands, strain, nullptr, out4), "dd_solve_strain");
  c.nodes = ddg_solver_nodes(c.solver);
}

// Same, each declarer's NS tricks found by stepping from the seed ns4[declarer].
inline void dd_solve_strain_guess(DDCtx& c, const uint64_t* hands, int strain, const int* ns4, int* out4) {
  check(ddg_solve_strain(c.solver, hands, strain, ns4, out4), "dd_solve_strain_guess");
  c.nodes = ddg_solver_nodes(c.solver);
}

// NS tricks with `leader` on lead in the context's deal and trump: binary search whose
// first target is `guess`.
inline int dd_ns_tricks(DDCtx& c, int leader, int guess) {
  int ns = 0;
  check(ddg_ns_tricks(c.solver, c.hand, dd_suit_strain(c.trump), leader, guess, 0, &ns), "dd_ns_tricks");
  c.nodes = ddg_solver_nodes(c.solver);
  return ns;
}

// The same, stepping up or down from `guess` (a right guess costs two searches).
inline int dd_ns_tricks_from(DDCtx& c, int leader, int guess) {
  int ns = 0;
  check(ddg_ns_tricks(c.solver, c.hand, dd_suit_strain(c.trump), leader, guess, 1, &ns), "dd_ns_tricks_from");
  c.nodes = ddg_solver_nodes(c.solver);
  return ns;
}

// All 20 results of n deals in one launch: out20[i*20 + strain*4 + declarer].
inline void dd_solve_deals(DDCtx& c, const uint64_t* hands, int64_t n, uint8_t* out20) {
  ddg_stats st;
  check(ddg_solve_batch(c.solver, hands, n, out20, &st), "ddg_solve_batch");
  c.nodes = ddg_solver_nodes(c.solver);
}

}  // namespace ddg
