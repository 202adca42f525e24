// Host-only checks of index arithmetic the particle kernels rely on
// (csrc/particles.cuh, csrc/common.cuh):
//   * class_ord is a bijection of the 512 tile-local cells onto 0..511,
//     class-major in bucket order (the bucket of a cell is 8 tile + class),
//     and inside each class it follows the cell's linear index;
//   * the multiply-shift division FastDiv and decode_cell give exact
//     quotients for every cell index of every supported grid size, and
//     FastDiv for 32-bit dividends across the whole range.
// Prints "ok" or the first violation.
#include <cstdio>

#include "common.cuh"
#include "particles.cuh"

int main()
{
    using namespace gev;
    int seen[512] = {0};
    int ord_of[512];
    const int N = 16, nt = 2;
    for (int z = 0; z < 8; z++)
        for (int y = 0; y < 8; y++)
            for (int x = 0; x < 8; x++) {
                const int o = class_ord(x, y, z);
                if (o < 0 || o >= 512 || seen[o]++) { printf("not a bijection at (%d,%d,%d): %d\n", x, y, z, o); return 1; }
                ord_of[x + 8 * (y + 8 * z)] = o;
            }
    // for every pair of cells of one tile: rank order == (bucket, linear cell index) order
    for (int a = 0; a < 512; a++)
        for (int b = 0; b < 512; b++) {
            const int ax = a % 8, ay = (a / 8) % 8, az = a / 64, bx = b % 8, by = (b / 8) % 8, bz = b / 64;
            // the tile at (1, 0, 1) of a 16^3 grid: bucket of the global cell
            const unsigned ba = bucket_of_cell(N, nt, 8 + ax, ay, 8 + az), bb = bucket_of_cell(N, nt, 8 + bx, by, 8 + bz);
            const bool rank_less = ord_of[a] < ord_of[b];
            const bool key_less = ba < bb || (ba == bb && a < b);
            if (rank_less != key_less) { printf("order differs for cells %d and %d\n", a, b); return 1; }
        }
    const int sizes[] = {16, 32, 64, 128, 256, 384, 512, 768};
    for (int n : sizes) {
        const FastDiv f((uint32_t)n);
        const uint32_t n3 = (uint32_t)n * n * n;
        for (uint32_t c = 0; c < n3; c++) {
            int x, y, z;
            decode_cell(c, f, x, y, z);
            if ((uint32_t)x != c % n || (uint32_t)y != (c / n) % n || (uint32_t)z != c / ((uint32_t)n * n)) {
                printf("decode_cell(%u) wrong for N = %d\n", c, n);
                return 1;
            }
        }
        for (uint64_t v = 0; v <= 0xffffffffull; v += 65521) {   // a prime stride over the 32-bit range
            if (f.div((uint32_t)v) != (uint32_t)v / (uint32_t)n) { printf("div(%llu) wrong for N = %d\n", (unsigned long long)v, n); return 1; }
        }
        if (f.div(0xffffffffu) != 0xffffffffu / (uint32_t)n) { printf("div(max) wrong for N = %d\n", n); return 1; }
    }
    printf("ok\n");
    return 0;
}
