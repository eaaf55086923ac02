// Host driver for the tile lists of the grouped GEMM (exciting_b200/csrc/zgemm.cu),
// used by tests/test_group_tiles.py.  Reads one product per line from stdin,
//   m n k uplo_c tri_a tri_b
// appends each to one launch's lists with zgemm_group_add (tile rows from
// argv[1]), orders the launch with zgemm_group_order and prints one tile per
// line: product, row tile, column tile, K range.  Host code only.
#include <cstdio>
#include <cstdlib>

#include "zgemm.cu"

void count_launch(int) {}
void excfv_set_error(const char*, ...) {}

int main(int argc, char** argv) {
  const int tbm = argc > 1 ? std::atoi(argv[1]) : 64;
  std::vector<ZgemmArgs> probs;
  std::vector<GroupTile> tiles;
  int m, n, k, uplo, ta, tb;
  while (std::scanf("%d %d %d %d %d %d", &m, &n, &k, &uplo, &ta, &tb) == 6) {
    ZgemmArgs a{};
    a.m = m; a.n = n; a.k = k; a.alpha = cmk(1.0, 0.0); a.beta = cmk(0.0, 0.0);
    a.batch = 1; a.uplo_c = uplo; a.tri_a = ta; a.tri_b = tb; a.splitk = 1;
    zgemm_group_add(a, probs, tiles, tbm);
  }
  zgemm_group_order(tiles, 0);
  std::printf("%zu\n", probs.size());
  for (const GroupTile& t : tiles) std::printf("%d %d %d %lld\n", t.prob, t.ti, t.tj, t.klen);
  return 0;
}
