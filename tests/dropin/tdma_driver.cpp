// Calls MACSolver2DAxisym::SolveTDMA of the drop-in class (a host method: no
// GPU is touched) on a batch of tridiagonal systems.
//
// usage: tdma_driver <in.bin> <out.bin>
//   in.bin:  int32 n, count; per system float64 a[n], b[n], c[n], d[n]
//   out.bin: per system int32 status, float64 c[n], d[n] as SolveTDMA leaves them
#include <cstdint>
#include <cstdio>
#include <vector>

#include "mac2dAxisym.h"

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE *fi = std::fopen(argv[1], "rb");
    FILE *fo = std::fopen(argv[2], "wb");
    if (!fi || !fo) return 2;
    int32_t hdr[2];
    if (std::fread(hdr, sizeof(int32_t), 2, fi) != 2) return 2;
    const int n = hdr[0], count = hdr[1];
    MACSolver2DAxisym solver(1000.0, 1.226, 1.0e-3, 1.78e-5, 9.8, GAXISENUM2DAXISYM::Z, 1.0, 1.0, 0.0728, 8, 8, 0.0,
                             0.0, 0.5, 1.0, 0.3, 1.0, 1, 1, 3, false);
    std::vector<double> a(n), b(n), c(n), d(n);
    for (int s = 0; s < count; s++) {
        for (std::vector<double> *v : {&a, &b, &c, &d})
            if (std::fread(v->data(), sizeof(double), n, fi) != (size_t)n) return 2;
        const int32_t rc = solver.SolveTDMA(a, b, c, d, n);
        std::fwrite(&rc, sizeof rc, 1, fo);
        std::fwrite(c.data(), sizeof(double), n, fo);
        std::fwrite(d.data(), sizeof(double), n, fo);
    }
    std::fclose(fi);
    std::fclose(fo);
    return 0;
}
