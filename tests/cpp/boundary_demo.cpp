// boundary_demo.cpp -- a reference-style C++ caller of the B200 path through
// include/dda_cuda.hpp only (dda::CudaMatVec<T>, dda::CudaSolver<T>), the way
// DDA/DDAMain.cpp drives MatVec<T> and IterativeSolverBase<T>.
//
//   boundary_demo <out.bin>
//
// Target: sphere of radius 0.5 um, grid unit 0.1 um, m = 1.5+0.1i, lambda
// 1 um, propagation (0,0,1), LDR.  Writes, as raw little-endian doubles:
// nvs, the FP64 matvec of a fixed input x_i = (sin i, cos 2i) (3*nvs complex),
// the FP32 matvec of the same input, and the FP64 QMR-CS polarisation of
// polarisation 1 at relative residual 1e-8 followed by its iteration count.
// Exits 2 with the error message when the library reports an error (for
// instance: no CUDA device).
#include <cmath>
#include <complex>
#include <cstdio>
#include <vector>

#include "dda_cuda.hpp"

int main(int argc, char** argv) {
  if (argc != 2) {
    std::fprintf(stderr, "usage: boundary_demo <out.bin>\n");
    return 1;
  }
  try {
    dda_geometry* g = nullptr;
    if (dda_geom_sphere("0.5um", "0.1um", &g) != 0) throw dda::Error(-1, dda_frontend_error());
    const uint32_t nv = dda_geom_nv(g);
    uint32_t box[3];
    dda_geom_box_size(g, box);
    double lambda = 0, d = dda_geom_grid_unit(g);
    dda_parse_length_m("1um", &lambda);
    const double k = 2 * std::acos(-1.0) / lambda;
    dda_problem p = {};
    p.nv = nv;
    for (int a = 0; a < 3; a++) {
      p.box[a] = box[a];
      p.grid[a] = dda_fft_fit(2 * box[a], 0, 1);  // DDAParams: fftFit(2 box)
    }
    p.positions = dda_geom_positions(g);
    p.materials = dda_geom_materials(g);
    p.nmat = 1;
    p.kd = k * d;
    p.grid_unit = d;
    p.max_rhs = 1;
    const double refr[6] = {1.5, 0.1, 1.5, 0.1, 1.5, 0.1};
    const double prop[3] = {0, 0, 1};
    std::vector<std::complex<double>> cc(3), ccs(3), chi(3);
    if (dda_couple_constants(DDA_POL_LDR, 1, refr, d, k, prop, 1, (double*)cc.data(), (double*)ccs.data(),
                             (double*)chi.data()) != 0)
      throw dda::Error(-1, dda_frontend_error());

    dda::CudaMatVec<double> mv64(p);
    dda::CudaMatVec<float> mv32(p);
    mv64.setCoupleConstants(ccs);
    mv32.setCoupleConstants(ccs);
    const size_t nvs = mv64.vecStride(), n = 3 * nvs;
    std::vector<std::complex<double>> x(n, 0.0), y64;
    std::vector<std::complex<float>> x32(n), y32;
    for (size_t c = 0; c < 3; c++)
      for (size_t i = 0; i < nv; i++) {
        const size_t j = c * nvs + i;
        x[j] = std::complex<double>(std::sin((double)j), std::cos(2.0 * j));
      }
    for (size_t j = 0; j < n; j++) x32[j] = std::complex<float>(x[j]);
    mv64.apply(x, y64, false);
    mv32.apply(x32, y32, false);

    std::vector<std::complex<double>> einc(n);
    if (dda_einc_plane(g, k, prop, 1, (double*)einc.data()) != 0) throw dda::Error(-1, dda_frontend_error());
    dda::CudaSolver<double> solver(mv64, "qmr");
    std::vector<double> residuals;
    std::vector<std::complex<double>> pol = solver.getPolVec(einc, 1e-8, &residuals);
    // the --ftype float vectors: CudaSolver<float> on the FP32 context
    std::vector<std::complex<float>> einc32(einc.begin(), einc.end());
    dda::CudaSolver<float> solver32(mv32, "bicgstab");
    std::vector<std::complex<float>> pol32 = solver32.getPolVec(einc32, 1e-5f);
    dda_geom_free(g);

    std::FILE* f = std::fopen(argv[1], "wb");
    if (!f) throw dda::Error(-1, "cannot open output");
    const double hdr = (double)nvs;
    std::fwrite(&hdr, sizeof hdr, 1, f);
    std::fwrite(y64.data(), sizeof(y64[0]), n, f);
    std::vector<std::complex<double>> y32d(y32.begin(), y32.end());
    std::fwrite(y32d.data(), sizeof(y32d[0]), n, f);
    std::fwrite(pol.data(), sizeof(pol[0]), n, f);
    const double iters = (double)solver.stats()[0].iterations;
    std::fwrite(&iters, sizeof iters, 1, f);
    std::vector<std::complex<double>> pol32d(pol32.begin(), pol32.end());
    std::fwrite(pol32d.data(), sizeof(pol32d[0]), n, f);
    std::fclose(f);
    std::printf("ok %zu %lld %zu\n", nvs, (long long)solver.stats()[0].iterations, residuals.size());
    return 0;
  } catch (const dda::Error& e) {
    std::fprintf(stderr, "dda::Error %d: %s\n", e.code, e.what());
    return 2;
  }
}
