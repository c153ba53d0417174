// Host-side split of row/column 2-factors into the canonical P/Q pair
// (src/no_three_75/state.py:47-85, points_to_permutations): P is the perfect
// matching that augmenting paths find when the rows are taken in order and each
// row's two columns in ascending order; Q takes each row's other column.  The
// search order is the reference's, so the same points give the same P/Q.  Plain
// C on the host: the beam searches call it on their reported elites, where the
// interpreted version took about 270 us per n = 75 state.
#include <stdint.h>
#include <string.h>

#include "n3_common.cuh"

namespace n3host {
namespace {

struct Matcher {
  int n;
  int adj[N3_MAX_N][2];
  int owner[N3_MAX_N];  // column -> row matched through P
  bool seen[N3_MAX_N];

  bool augment(int row) {
    for (int k = 0; k < 2; ++k) {
      const int col = adj[row][k];
      if (seen[col]) continue;
      seen[col] = true;
      if (owner[col] == -1 || augment(owner[col])) {
        owner[col] = row;
        return true;
      }
    }
    return false;
  }
};

}  // namespace
}  // namespace n3host

extern "C" int n3_normalize_pairs(const int32_t* p, const int32_t* q, int B, int n, int32_t* p_out, int32_t* q_out) {
  if (B < 0 || n < 2 || n > N3_MAX_N) return n3host::set_error(N3_ERR_RANGE, "normalize_pairs: bad sizes B=%d n=%d", B, n);
  if (B > 0 && (!p || !q || !p_out || !q_out)) return n3host::set_error(N3_ERR_ARG, "normalize_pairs: null pointer");
  n3host::Matcher m;
  m.n = n;
  for (int b = 0; b < B; ++b) {
    const int32_t* pb = p + (size_t)b * n;
    const int32_t* qb = q + (size_t)b * n;
    int degree[N3_MAX_N];
    memset(degree, 0, sizeof(degree));
    for (int r = 0; r < n; ++r) {
      const int a = pb[r], c = qb[r];
      if (a < 0 || a >= n || c < 0 || c >= n || a == c)
        return n3host::set_error(N3_ERR_ARG, "normalize_pairs: state %d is not a row/column 2-factor (row %d)", b, r);
      m.adj[r][0] = a < c ? a : c;
      m.adj[r][1] = a < c ? c : a;
      ++degree[a];
      ++degree[c];
    }
    for (int c = 0; c < n; ++c)
      if (degree[c] != 2)
        return n3host::set_error(N3_ERR_ARG, "normalize_pairs: state %d is not a row/column 2-factor (column %d)", b, c);
    for (int c = 0; c < n; ++c) m.owner[c] = -1;
    for (int r = 0; r < n; ++r) {
      for (int c = 0; c < n; ++c) m.seen[c] = false;
      if (!m.augment(r)) return n3host::set_error(N3_ERR_ARG, "normalize_pairs: state %d has no perfect matching", b);
    }
    int32_t* po = p_out + (size_t)b * n;
    int32_t* qo = q_out + (size_t)b * n;
    for (int c = 0; c < n; ++c) po[m.owner[c]] = c;
    for (int r = 0; r < n; ++r) qo[r] = m.adj[r][0] == po[r] ? m.adj[r][1] : m.adj[r][0];
  }
  return N3_OK;
}
