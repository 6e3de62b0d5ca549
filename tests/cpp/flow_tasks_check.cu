// Host-only check of the flag-ordered sweeps' task lists (no GPU needed): for
// random levels of fronts, flow_tasks lists every forward task (front, row
// block) and every backward task (front, pivot block) exactly once, the flag
// offsets give each front its pivot blocks, and every flag a task waits for is
// raised by a task listed before it.  The last property is what keeps the
// persistent grid from stalling: a CTA takes its tasks in list order, so the
// earliest unfinished task always has its dependencies done.
#include <cstdio>
#include <random>
#include <vector>

#include "../../updating-multifrontal_b200/csrc/kernels_solve.cu"

namespace mfgpu {
std::atomic<long long> g_launches{0};
}
using namespace mfgpu;

int main() {
  std::mt19937 rng(20261204);
  long long checked = 0;
  for (int trial = 0; trial < 3000; trial++) {
    const int nf = 1 + (int)(rng() % 12);
    std::vector<int> n(nf), N(nf);
    for (int i = 0; i < nf; i++) {
      n[i] = (int)(rng() % 2000);                    // empty pivot sets included
      N[i] = n[i] + (int)(rng() % 3000);
    }
    std::vector<int> fwd, bwd, flagoff;
    flow_tasks(n, N, fwd, bwd, flagoff);
    auto fail = [&](const char* what) {
      printf("%s (trial %d)\n", what, trial);
      return 1;
    };
    if ((int)flagoff.size() != nf + 1 || flagoff[0] != 0) return fail("flag offsets");
    std::vector<int> nb(nf), rb(nf);
    for (int i = 0; i < nf; i++) {
      nb[i] = (n[i] + 63) / 64;
      rb[i] = nb[i] + (N[i] - n[i] + 63) / 64;
      if (flagoff[i + 1] - flagoff[i] != nb[i]) return fail("flags per front");
    }
    // forward: (i, R) waits for pivot blocks j < min(R, nb) of front i
    std::vector<std::vector<int>> seen(nf);
    for (int i = 0; i < nf; i++) seen[i].assign(rb[i], 0);
    for (size_t p = 0; p + 1 < fwd.size(); p += 2) {
      const int i = fwd[p], R = fwd[p + 1];
      if (i < 0 || i >= nf || R < 0 || R >= rb[i] || seen[i][R]) return fail("forward task");
      for (int j = 0; j < std::min(R, nb[i]); j++)
        if (!seen[i][j]) return fail("forward wait on a later task");
      seen[i][R] = 1;
      checked++;
    }
    for (int i = 0; i < nf; i++)
      for (int R = 0; R < rb[i]; R++)
        if (!seen[i][R]) return fail("forward task missing");
    // backward: (i, j) waits for pivot blocks R > j of front i
    for (int i = 0; i < nf; i++) seen[i].assign(nb[i], 0);
    for (size_t p = 0; p + 1 < bwd.size(); p += 2) {
      const int i = bwd[p], j = bwd[p + 1];
      if (i < 0 || i >= nf || j < 0 || j >= nb[i] || seen[i][j]) return fail("backward task");
      for (int R = j + 1; R < nb[i]; R++)
        if (!seen[i][R]) return fail("backward wait on a later task");
      seen[i][j] = 1;
      checked++;
    }
    for (int i = 0; i < nf; i++)
      for (int j = 0; j < nb[i]; j++)
        if (!seen[i][j]) return fail("backward task missing");
  }
  printf("ok %lld tasks\n", checked);
  return 0;
}
