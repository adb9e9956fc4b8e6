// Test infrastructure: a C++ caller written against the reference's header-level solve API
// shape (include/dd_solve.hpp over libddg.so), the way a caller of hsperr/dds_gpu's
// src/dd.h would port its code. It solves the deals of DEALS.bin (32-byte records) through
// every call of the header and prints one JSON object of the results, which the GPU tests
// compare with the reference's golden tables and node counts:
//   strain   dd_solve_strain per (deal, strain)           -> 20 results per deal
//   guess    dd_solve_strain_guess with seeds 7            -> 20 results per deal
//   ns       dd_ns_tricks per (deal, strain, leader)      -> 20 results per deal (declarer order)
//   ns_from  dd_ns_tricks_from per (deal, strain, leader) -> 20 results per deal
//   deals    dd_solve_deals over all deals                 -> 20 results per deal
//   strain_nodes  the search nodes of each dd_solve_strain call (DDCtx::nodes deltas)
//
//   dd_solve_caller DEALS.bin
#include <stdio.h>

#include <vector>

#include "dd_solve.hpp"

static void print_list(const char* name, const std::vector<long long>& v, bool last = false) {
  printf("\"%s\": [", name);
  for (size_t i = 0; i < v.size(); i++) printf("%s%lld", i ? ", " : "", v[i]);
  printf("]%s", last ? "" : ", ");
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s DEALS.bin\n", argv[0]);
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 1;
  std::vector<uint64_t> hands;
  uint64_t rec[4];
  while (fread(rec, 8, 4, f) == 4) hands.insert(hands.end(), rec, rec + 4);
  fclose(f);
  const long n = (long)hands.size() / 4;
  std::vector<long long> strain, guess, ns, ns_from, deals, strain_nodes;
  try {
    ddg::DDCtx c(10);
    for (long i = 0; i < n; i++) {
      const uint64_t* h = hands.data() + i * 4;
      for (int st = 0; st < 5; st++) {
        int out4[4];
        const uint64_t before = c.nodes;
        ddg::dd_solve_strain(c, h, st, out4);
        strain_nodes.push_back((long long)(c.nodes - before));
        for (int d = 0; d < 4; d++) strain.push_back(out4[d]);
      }
      for (int st = 0; st < 5; st++) {
        int seeds[4] = {7, 7, 7, 7}, out4[4];
        ddg::dd_solve_strain_guess(c, h, st, seeds, out4);
        for (int d = 0; d < 4; d++) guess.push_back(out4[d]);
      }
      for (int k = 0; k < 4; k++) c.hand[k] = h[k];
      for (int st = 0; st < 5; st++) {
        c.trump = ddg::dd_strain_suit(st);
        ddg::dd_next_gen(c);
        for (int d = 0; d < 4; d++) {
          const int leader = (d + 1) & 3;
          const int a = ddg::dd_ns_tricks(c, leader, 7);
          const int b = ddg::dd_ns_tricks_from(c, leader, 7);
          ns.push_back((d & 1) == 0 ? a : 13 - a);
          ns_from.push_back((d & 1) == 0 ? b : 13 - b);
        }
      }
    }
    std::vector<uint8_t> out20((size_t)n * 20);
    ddg::dd_solve_deals(c, hands.data(), n, out20.data());
    for (uint8_t v : out20) deals.push_back(v);
    printf("{");
    print_list("strain", strain);
    print_list("guess", guess);
    print_list("ns", ns);
    print_list("ns_from", ns_from);
    print_list("deals", deals);
    print_list("strain_nodes", strain_nodes, true);
    printf("}\n");
  } catch (const ddg::Error& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
