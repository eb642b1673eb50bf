// Drop-in for `TransferDisStream <yfile> <xfile> <outprefix> <ntip>`
// (cu/TransferDisStream.cu:130-344), on one GPU: writes <outprefix>_ymin.bin
// and <outprefix>_xmin.bin ({2, n} + min distance + clade size per row).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "casphy.h"
#include "toolio.h"

int main(int argc, char* argv[]) {
    setbuf(stdout, nullptr);
    if (argc < 5) {
        printf("Error: no sufficient args.\n");
        return argc < 3 ? 0 : 1;
    }
    const double t0 = tool::now_s();
    const uint32_t ntip = (uint32_t)atoi(argv[4]);
    uint32_t ny = 0, ncol = 0, nx = 0, ncolx = 0;
    std::vector<uint32_t> y, x;
    if (!tool::read_mat(argv[1], ny, ncol, y) || !tool::read_mat(argv[2], nx, ncolx, x)) {
        fprintf(stderr, "TransferDisStream: cannot open input\n");
        return 1;
    }
    // the x file is read with the y file's column count
    if (ncolx != ncol) {
        FILE* f = fopen(argv[2], "rb");
        uint32_t dim[2];
        if (fread(dim, sizeof(uint32_t), 2, f) != 2) dim[0] = 0;
        x.assign((size_t)nx * ncol, 0u);
        if (!x.empty()) {
            size_t got = fread(x.data(), sizeof(uint32_t), x.size(), f);
            (void)got;
        }
        fclose(f);
    }
    const int dev = tool::pick_device();
    if (dev < 0) return tool::fail("TransferDisStream", CASPHY_ENODEV);
    printf("calculate crossXOR between 1st mat with %d rows and 2nd mat with %d rows.\n", (int)ny, (int)nx);
    std::vector<uint32_t> ymin(ny + 1), ysize(ny + 1), xmin(nx + 1), xsize(nx + 1);
    int rc = casphy_transfer_dis(ny, nx, ncol, ntip, y.data(), x.data(), ymin.data(), ysize.data(), xmin.data(),
                                 xsize.data());
    if (rc) return tool::fail("TransferDisStream", rc);
    printf("Running time on GPU: %.5fs\n", tool::now_s() - t0);
    std::vector<uint32_t> yb(ymin.begin(), ymin.begin() + ny), xb(xmin.begin(), xmin.begin() + nx);
    yb.insert(yb.end(), ysize.begin(), ysize.begin() + ny);
    xb.insert(xb.end(), xsize.begin(), xsize.begin() + nx);
    const std::string out = argv[3];
    if (!tool::write_mat(out + "_ymin.bin", 2, ny, yb.data(), yb.size()) ||
        !tool::write_mat(out + "_xmin.bin", 2, nx, xb.data(), xb.size()))
        return 1;
    return 0;
}
