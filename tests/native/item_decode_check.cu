// Host-side check of the tensor-core engine's work-item decode (decode_item in
// global_tc.cu is host-callable): prints every non-empty item of a schedule as
// "column_tile first_row_block end_row_block", for comparison with
// sred_b200.clutils.decode_items. Usage: item_decode_check n bn panel sms
// (panel 0 = one panel). Built and run by tests/test_item_decode.py.
#include "../../sred_b200/csrc/global_tc.cu"

#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
  using namespace sred;
  if (argc != 5) return 2;
  const int n = std::atoi(argv[1]), bn = std::atoi(argv[2]), panel = std::atoi(argv[3]), sms = std::atoi(argv[4]);
  TcArgs g{};
  g.n_rb = (n + kBM - 1) / kBM;
  g.n_ct = (n + bn - 1) / bn;
  int L = 0;
  const long long items = gram_tc_items(n, bn, &L, sms, 0);
  g.L = L;
  g.h = L / (bn / kBM);
  g.n_runs = (g.n_rb + L - 1) / L;
  g.panel = panel > 0 ? panel : g.n_ct;
  g.n_panels = (g.n_ct + g.panel - 1) / g.panel;
  g.ec.n = n;
  for (long long it = 0; it < items; it++) {
    int ct, rb0, rb1;
    if (decode_item(it, g, bn / kBM, ct, rb0, rb1)) std::printf("%d %d %d\n", ct, rb0, rb1);
  }
  // Each CTA's cursor (start at its first item, step by the grid) visits the
  // items decode_item gives, and its two passes split each item's row blocks.
  int bad = 0;
  for (int grid : {148, 7, 1}) {
    g.item0 = 0;
    g.item1 = items;
    for (int b = 0; b < grid; b++) {
      ItemCursor cur;
      cur.init(g, b);
      for (; cur.it < items; cur.advance(g, grid)) {
        int ct, rb0, rb1, c0, lo0, hi0, c1, lo1, hi1;
        const bool any = decode_item(cur.it, g, bn / kBM, ct, rb0, rb1);
        const bool p0 = cur.part(g, bn / kBM, bn, 0, c0, lo0, hi0);
        const bool p1 = cur.part(g, bn / kBM, bn, 1, c1, lo1, hi1);
        const bool same = c0 == ct && c1 == ct && lo0 == rb0 && hi0 == lo1 && hi1 == rb1 && any == (p0 || p1);
        if (!same) bad++;
      }
    }
  }
  std::printf("cursor %s\n", bad ? "MISMATCH" : "ok");
  return 0;
}
