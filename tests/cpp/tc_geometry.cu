// Host-only check of the tensor-core update's tile bookkeeping (no GPU
// needed): for many fronts, panels [K, K + w) and column bounds, the tile
// count per front, the decoding of a tile index into (block row, block
// column) - a bijection onto the tile set, in the grouped order - and the pack
// capacity agree with a brute-force enumeration of the 128 x 256 tiles of
// C(k1:N, k1:cmax) that touch its lower triangle.
#include <cstdio>
#include <random>
#include <set>
#include <utility>

#include "../../updating-multifrontal_b200/csrc/kernels_tc.cu"

namespace mfgpu {
std::atomic<long long> g_launches{0};
}
using namespace mfgpu;

int main() {
  std::mt19937 rng(20261203);
  long long checked = 0;
  for (int trial = 0; trial < 20300; trial++) {
    // the last 300 trials: fronts of up to 50,000 (several row groups of tiles)
    const int span = trial < 20000 ? 3000 : 25000;
    const int n = 1 + (int)(rng() % span), N = n + (int)(rng() % span);
    const int w = (rng() % 2) ? 512 : 128;
    const int K = (int)(rng() % ((n + w - 1) / w + 1)) * w;
    const int cend = (rng() % 3 == 0) ? -1 : K + 512 * (1 + (int)(rng() % 2));
    const PanelGeo g = panel_geo(n, N, K, w, cend);
    // brute force: block rows of 128 from k1, block columns of 256 from k1,
    // tiles holding an entry (r, c) with k1 <= c < cmax, c <= r < N
    std::set<std::pair<int, int>> want;
    if (K < n) {
      const int k1 = std::min(K + w, n), cmax = cend < 0 ? N : std::min(cend, n);
      for (int I = 0; k1 + 128 * I < N; I++)
        for (int J = 0; k1 + 256 * J < cmax && 256 * J <= 128 * I + 127; J++) want.insert({I, J});
      if (!(g.nb == 0 ? want.empty() : g.k1 == k1 && g.cmax == cmax)) {
        printf("geometry mismatch n=%d N=%d K=%d w=%d cend=%d\n", n, N, K, w, cend);
        return 1;
      }
    }
    const int T = geo_tiles(g);
    if (T != (int)want.size()) {
      printf("count mismatch n=%d N=%d K=%d w=%d cend=%d: %d vs %zu\n", n, N, K, w, cend, T, want.size());
      return 1;
    }
    std::set<std::pair<int, int>> got;
    for (int t = 0; t < T; t++) {
      int I, J;
      tile_ij(t, g.nb, g.nj, I, J);
      got.insert({I, J});
    }
    if (got != want) {
      printf("decode mismatch n=%d N=%d K=%d w=%d cend=%d\n", n, N, K, w, cend);
      return 1;
    }
    const std::vector<int> nv{n}, Nv{N};
    const PanelGeo gp = panel_geo(n, N, K, w, -1);   // the pack covers every row block below k1
    if (tc_tiles(nv, Nv, K, w, cend) != T || tc_pack_cap(nv, Nv, K, w) != gp.nb * gp.nch ||
        (T > 0 && (gp.nb != g.nb || gp.nch != g.nch))) {
      printf("host totals mismatch n=%d N=%d K=%d w=%d cend=%d\n", n, N, K, w, cend);
      return 1;
    }
    checked += T;
  }
  printf("ok %lld tiles\n", checked);
  return 0;
}
