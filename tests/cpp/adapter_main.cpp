// Test driver of the C++ adapter (include/stpgpu_stp.hpp): images a
// snapshot through stp::ImageVisibilities and through the template
// stp::image_visibilities with a functor object, then runs
// stp::SourceFindImage on the image, writing the results for the Python test
// to compare with the CPU oracle.
//
//   adapter_main <input.bin> <output prefix>
//
// input.bin: int64 n; int32 image_size, kernel_function, kernel_support,
// oversampling, kernel_exact, analytic_gcf, num_wplanes, max_wpconv_support;
// double cell_size, kernel_trunc_perc; then vis (n complex128), weights (n),
// uvw (n x 3 column-major).
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "stp_shim.h"
#include "stpgpu_stp.hpp"

template <typename T>
static void read_into(std::FILE* f, T* p, size_t n)
{
    if (n && std::fread(p, sizeof(T), n, f) != n)
        throw std::runtime_error("short read");
}

template <typename T>
static void write_file(const std::string& path, const T* p, size_t n)
{
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(p, sizeof(T), n, f) != n)
        throw std::runtime_error("cannot write " + path);
    std::fclose(f);
}

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input.bin output_prefix\n", argv[0]);
        return 2;
    }
    try {
        std::FILE* f = std::fopen(argv[1], "rb");
        if (!f)
            throw std::runtime_error("cannot open input");
        int64_t n = 0;
        int32_t iv[8];
        double dv[2];
        read_into(f, &n, 1);
        read_into(f, iv, 8);
        read_into(f, dv, 2);
        arma::cx_mat vis(size_t(n), 1);
        arma::mat weights(size_t(n), 1), uvw(size_t(n), 3);
        read_into(f, reinterpret_cast<double*>(vis.memptr()), size_t(2 * n));
        read_into(f, weights.memptr(), size_t(n));
        read_into(f, uvw.memptr(), size_t(3 * n));
        std::fclose(f);

        stp::ImagerPars ip(unsigned(iv[0]), dv[0], 1.0, stp::KernelFunction(iv[1]), unsigned(iv[2]), iv[4] != 0,
            unsigned(iv[3]), true, true, iv[5] != 0);
        stp::W_ProjectionPars wp;
        wp.num_wplanes = unsigned(iv[6]);
        wp.max_wpconv_support = unsigned(iv[7]);
        wp.kernel_trunc_perc = dv[1];
        const std::string out = argv[2];

        // the class path: functor chosen from img_pars.kernel_function
        stp::ImageVisibilities iv_result(vis, weights, uvw, ip, wp);
        write_file(out + "_image.bin", iv_result.vis_grid.memptr(), iv_result.vis_grid.n_elem);
        write_file(out + "_beam.bin", iv_result.sampling_grid.memptr(), iv_result.sampling_grid.n_elem);

        // the template path with a functor object (A-projection parameters defaulted)
        stp::ImagerPars ip2 = ip;
        ip2.generate_beam = false;
        auto r = stp::image_visibilities(stp::GaussianSinc(double(iv[2])), vis, weights, uvw, ip2, wp);
        write_file(out + "_image_gs.bin", r.first.memptr(), r.first.n_elem);
        if (!r.second.is_empty())
            throw std::runtime_error("beam returned without generate_beam");

        // the source finder on the imaged map (reference defaults past the thresholds)
        stp::SourceFindImage sf(iv_result.vis_grid, 5.0, 3.0);
        write_file(out + "_labels.bin", sf.label_map.memptr(), sf.label_map.n_elem);
        std::FILE* g = std::fopen((out + "_islands.txt").c_str(), "w");
        std::fprintf(g, "%.17g %.17g\n", double(sf.bg_level), sf.rms_est);
        for (const auto& isl : sf.islands)
            std::fprintf(g, "%d %d %.17g %d %d %d %.17g %.17g %.17g %.17g %.17g %.17g\n", isl.label_idx, isl.sign,
                isl.extremum_val, isl.extremum_x_idx, isl.extremum_y_idx, isl.num_samples, isl.moments_fit.amplitude,
                isl.moments_fit.x_centre, isl.moments_fit.y_centre, isl.moments_fit.semimajor,
                isl.moments_fit.semiminor, isl.moments_fit.theta);
        std::fclose(g);

        // errors surface as std::runtime_error with the library's message
        try {
            stp::ImagerPars bad = ip;
            bad.cell_size = 0.0;
            stp::ImageVisibilities(vis, weights, uvw, bad, wp);
            std::fprintf(stderr, "expected an exception for cell_size 0\n");
            return 1;
        } catch (const std::runtime_error& e) {
            std::printf("error path ok: %s\n", e.what());
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "adapter_main: %s\n", e.what());
        return 1;
    }
    std::printf("adapter ok\n");
    return 0;
}
