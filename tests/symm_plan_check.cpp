// Host-side checks of the symmetric form's work plan (pair_symm_plan) and of
// its panel sizing (symm_panel_width, symm_layout) in libinti_b200.so: no
// device is touched.  Every unordered pair of node blocks (I <= J) must be
// covered by exactly one work item, each panel's items must lie in its
// source-block range, the per-panel row lists must point at their own
// items, and the panel widths must respect the partial budget.
#include <cstdint>
#include <cstdio>
#include <set>
#include <utility>
#include <vector>

namespace inti {
struct SymPanel {
  int item_off = 0, nitems = 0;
  int rowptr_off = 0, rowitems_off = 0, rows = 0;
  int col0 = 0, ncols = 0;
};
void pair_symm_plan(int64_t n, int tpt, int ch, int pcols, std::vector<int32_t>& table,
                    std::vector<SymPanel>& panels, int& nb, int& nitems);
int symm_panel_width(int64_t n, int tpt, int ch, int pb, double budget);
void symm_layout(int64_t n, int tpt, int ch, int pb, double budget, int& pcols, int& ch_eff);
}  // namespace inti

using namespace inti;

int main() {
  int bad = 0, cases = 0;
  for (int64_t n : {1, 7, 255, 256, 257, 5400, 6912, 100000})
    for (int tpt : {2, 4})
      for (int ch : {1, 3, 1000})
        for (int pc : {1, 2, 5, 1 << 20}) {
          ++cases;
          std::vector<int32_t> t;
          std::vector<SymPanel> P;
          int nb = 0, ni = 0;
          pair_symm_plan(n, tpt, ch, pc, t, P, nb, ni);
          std::set<std::pair<int, int>> seen;
          int maxn = 0, col = 0;
          for (const SymPanel& p : P) {
            maxn = p.nitems > maxn ? p.nitems : maxn;
            if (p.col0 != col) ++bad;  // panels tile the source blocks in order
            col = p.col0 + p.ncols;
            if (p.rowitems_off + p.nitems > (int)t.size()) { ++bad; continue; }
            const int32_t* it = t.data() + p.item_off;
            const int32_t* rp = t.data() + p.rowptr_off;
            const int32_t* ri = t.data() + p.rowitems_off;
            if (p.rows != (nb < p.col0 + p.ncols ? nb : p.col0 + p.ncols)) ++bad;
            if (rp[0] != 0 || rp[p.rows] != p.nitems) ++bad;
            for (int q = 0; q < p.nitems; ++q) {
              const int I = it[3 * q], J0 = it[3 * q + 1], J1 = it[3 * q + 2];
              if (I < 0 || I >= p.rows || J0 < I || J0 < p.col0 || J1 > p.col0 + p.ncols || J1 <= J0) ++bad;
              for (int J = J0; J < J1; ++J)
                if (!seen.insert({I, J}).second) ++bad;
            }
            for (int B = 0; B < p.rows; ++B)
              for (int k = rp[B]; k < rp[B + 1]; ++k)
                if (it[3 * ri[k]] != B) ++bad;
          }
          if (col != nb) ++bad;
          if ((long)seen.size() != (long)nb * (nb + 1) / 2) ++bad;
          if (maxn != ni) ++bad;
        }
  // panel widths: the whole operator when it fits, otherwise within budget
  const int64_t n = 777600;
  const int w_all = symm_panel_width(n, 2, 650, 8, 64.0e9);
  const int w = symm_panel_width(n, 2, 650, 8, 2.0e9);
  if (w_all != (int)((n + 255) / 256)) ++bad;
  if (!(w >= 1 && w < w_all)) ++bad;
  int pcols = 0, ch_eff = 0;
  symm_layout(n, 2, 650, 8, 2.0e9, pcols, ch_eff);
  if (!(pcols >= 1 && ch_eff >= 1 && ch_eff <= pcols / 8 + 1)) ++bad;
  std::printf("%d plans checked, %d failures; N = %lld: %d of %d blocks per panel, %d per item\n", cases, bad,
              (long long)n, pcols, w_all, ch_eff);
  return bad != 0;
}
