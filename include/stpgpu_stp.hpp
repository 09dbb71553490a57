/*
 * stpgpu_stp.hpp -- C++ drop-in of the reference's imager and source-finder
 * entry points, over the C ABI of stpgpu.h.
 *
 *   stp::image_visibilities<T>(kernel_creator, vis, vis_weights, uvw_lambda,
 *                              img_pars, w_proj, a_proj)
 *       replaces src/stp/imager/imager.h:233-376 (same signature, same
 *       defaults, returns (image, beam));
 *   stp::ImageVisibilities(vis, vis_weights, uvw_lambda, img_pars, w_proj, a_proj)
 *       replaces src/stp/imager/imager.h:381-411 and src/stp/imager/imager.cpp:12-68
 *       (members vis_grid, sampling_grid);
 *   stp::IslandParams, stp::SourceFindImage(input_data, detection_n_sigma, ...)
 *       replace src/stp/sourcefind/sourcefind.h:63-133,143-201 (same
 *       constructor arguments and defaults; members label_map, islands,
 *       bg_level, rms_est, detection_n_sigma, analysis_n_sigma, fit_gaussian).
 *
 * Use: include this header where the reference includes imager.h and
 * sourcefind.h, after Armadillo and the reference's own stp/types.h
 * (real_t, ImagerPars, W_ProjectionPars, A_ProjectionPars, the enums),
 * stp/convolution/conv_func.h (the kernel functor classes),
 * stp/sourcefind/fitting.h (BoundingBox, Gaussian2dParams) and
 * stp/common/matstp.h (MatStp); drop imager.cpp and sourcefind.cpp from the
 * build and link libstpgpu.so.  Only these members of the containers are
 * used: memptr(), n_rows, n_cols, n_elem, set_size(rows, cols), reset().
 *
 * Semantics kept: column-major matrices; the image is unshifted (DC at
 * [0,0]); an all-zero sampling total returns empty matrices (imager.h:355);
 * the beam is empty unless generate_beam; errors throw std::runtime_error
 * (the reference's exception type, src/stp/common/fft.cpp:19-41) with the
 * library's message.  Arithmetic: FP64 when real_t is double (the plain
 * form, within 1e-10 of the reference's double build); compensated FP32
 * when real_t is float (the reference's USE_FLOAT build, within 1e-5).
 *
 * Differences to know: the kernel functor is identified by its type and
 * evaluated with truncation radius img_pars.kernel_support and the default
 * width normalisations -- exactly what ImageVisibilities builds
 * (imager.cpp:25-64) and every reference call site passes; a functor built
 * with another radius or widths is not read (its members are private).  The
 * FFT routine and wisdom file of ImagerPars are ignored (cuFFT).  The
 * intermediate per-label arrays of SourceFindImage (label_extrema_*) are
 * left empty; islands carry their values.  Calls run on CUDA device 0, or on
 * the device named by the STPGPU_DEVICE environment variable, through one
 * library context per host thread.
 */
#ifndef STPGPU_STP_HPP
#define STPGPU_STP_HPP

#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "stpgpu.h"

namespace stp {

namespace stpgpu_detail {

    // Kernel functor type -> stpgpu_kernel_function (enum values of src/stp/types.h:32-39).
    template <typename T>
    struct kernel_id;
    template <>
    struct kernel_id<TopHat> : std::integral_constant<int, STPGPU_TOPHAT> {
    };
    template <>
    struct kernel_id<Triangle> : std::integral_constant<int, STPGPU_TRIANGLE> {
    };
    template <>
    struct kernel_id<Sinc> : std::integral_constant<int, STPGPU_SINC> {
    };
    template <>
    struct kernel_id<Gaussian> : std::integral_constant<int, STPGPU_GAUSSIAN> {
    };
    template <>
    struct kernel_id<GaussianSinc> : std::integral_constant<int, STPGPU_GAUSSIANSINC> {
    };
    template <>
    struct kernel_id<PSWF> : std::integral_constant<int, STPGPU_PSWF> {
    };

    struct ContextDeleter {
        void operator()(stpgpu_context* c) const
        {
            if (c)
                stpgpu_destroy(c);
        }
    };

    // One context per host thread (a context serialises its calls on one
    // stream, as the reference's imager is not re-entrant either).
    inline stpgpu_context* context()
    {
        thread_local std::unique_ptr<stpgpu_context, ContextDeleter> ctx;
        if (!ctx) {
            int device = 0;
            if (const char* d = std::getenv("STPGPU_DEVICE"))
                device = std::atoi(d);
            stpgpu_context* c = nullptr;
            const stpgpu_status s = stpgpu_create(device, &c);
            if (s != STPGPU_OK)
                throw std::runtime_error("stpgpu_create failed with status " + std::to_string(int(s)));
            ctx.reset(c);
        }
        return ctx.get();
    }

    inline void check(stpgpu_context* c, stpgpu_status s)
    {
        if (s != STPGPU_OK)
            throw std::runtime_error(std::string(stpgpu_last_error(c)));
    }

    constexpr bool single = std::is_same<real_t, float>::value;

} // namespace stpgpu_detail

/* stp::image_visibilities, src/stp/imager/imager.h:233-376. */
template <typename T>
std::pair<arma::Mat<real_t>, arma::Mat<real_t>> image_visibilities(
    const T kernel_creator,
    const arma::cx_mat& vis,
    const arma::mat& vis_weights,
    const arma::mat& uvw_lambda,
    const ImagerPars& img_pars = ImagerPars(),
    const W_ProjectionPars& w_proj = W_ProjectionPars(),
    const A_ProjectionPars& a_proj = A_ProjectionPars())
{
    using namespace stpgpu_detail;
    (void)kernel_creator;
    const int64_t n = int64_t(vis.n_elem);
    if (int64_t(vis_weights.n_elem) != n || int64_t(uvw_lambda.n_rows) != n || uvw_lambda.n_cols != 3)
        throw std::runtime_error("image_visibilities: vis, vis_weights and uvw_lambda (n x 3) sizes disagree");
    stpgpu_imager_pars p {};
    p.image_size = int32_t(img_pars.image_size);
    p.padded_image_size = int32_t(img_pars.padded_image_size);
    p.cell_size = img_pars.cell_size;
    p.padding_factor = img_pars.padding_factor;
    p.kernel_function = kernel_id<T>::value;
    p.kernel_support = int32_t(img_pars.kernel_support);
    p.kernel_exact = img_pars.kernel_exact ? 1 : 0;
    p.oversampling = int32_t(img_pars.oversampling);
    p.generate_beam = img_pars.generate_beam ? 1 : 0;
    p.gridding_correction = img_pars.gridding_correction ? 1 : 0;
    p.analytic_gcf = img_pars.analytic_gcf ? 1 : 0;
    p.r_fft = 0;
    stpgpu_wproj_pars w {};
    w.num_wplanes = int32_t(w_proj.num_wplanes);
    w.max_wpconv_support = int32_t(w_proj.max_wpconv_support);
    w.undersampling_opt = int32_t(w_proj.undersampling_opt);
    w.kernel_trunc_perc = w_proj.kernel_trunc_perc;
    w.hankel_opt = w_proj.hankel_opt ? 1 : 0;
    w.hankel_proj_slice = w_proj.hankel_proj_slice ? 1 : 0;
    w.interp_type = int32_t(w_proj.interp_type);
    w.wplanes_median = w_proj.wplanes_median ? 1 : 0;
    stpgpu_aproj_pars a {};
    a.num_timesteps = int32_t(a_proj.num_timesteps);
    a.obs_dec = a_proj.obs_dec;
    a.obs_ra = a_proj.obs_ra;
    a.aproj_opt = a_proj.aproj_opt ? 1 : 0;
    a.aproj_mask_perc = a_proj.aproj_mask_perc;
    a.lha = a_proj.num_timesteps > 0 ? a_proj.lha.memptr() : nullptr;
    a.pbeam_coefs = a_proj.pbeam_coefs.empty() ? nullptr : a_proj.pbeam_coefs.data();
    a.n_pbeam_coefs = int32_t(a_proj.pbeam_coefs.size());

    const int size = int(img_pars.image_size);
    std::pair<arma::Mat<real_t>, arma::Mat<real_t>> out;
    out.first.set_size(size, size);
    if (img_pars.generate_beam)
        out.second.set_size(size, size);
    stpgpu_context* c = context();
    stpgpu_imager_info info {};
    check(c,
        stpgpu_image_visibilities_ex(c, vis.memptr(), STPGPU_C128, vis_weights.memptr(), uvw_lambda.memptr(), n, &p,
            &w, &a, single ? STPGPU_FP32C : STPGPU_FP64, out.first.memptr(),
            img_pars.generate_beam ? out.second.memptr() : nullptr, single ? STPGPU_F32 : STPGPU_F64, 0, &info));
    if (info.image_size == 0) { // zero sampling total: empty matrices (imager.h:355)
        out.first.reset();
        out.second.reset();
    }
    return out;
}

/* stp::ImageVisibilities, src/stp/imager/imager.h:381-411, imager.cpp:12-68:
 * the functor of img_pars.kernel_function with truncation kernel_support. */
class ImageVisibilities {
public:
    ImageVisibilities() = delete;
    ImageVisibilities(const arma::cx_mat& vis,
        const arma::mat& vis_weights,
        const arma::mat& uvw_lambda,
        const ImagerPars& img_pars = ImagerPars(),
        const W_ProjectionPars& w_proj = W_ProjectionPars(),
        const A_ProjectionPars& a_proj = A_ProjectionPars())
    {
        std::pair<arma::Mat<real_t>, arma::Mat<real_t>> r;
        const double s = double(img_pars.kernel_support);
        switch (img_pars.kernel_function) {
        case KernelFunction::TopHat:
            r = image_visibilities(TopHat(s), vis, vis_weights, uvw_lambda, img_pars, w_proj, a_proj);
            break;
        case KernelFunction::Triangle:
            r = image_visibilities(Triangle(s), vis, vis_weights, uvw_lambda, img_pars, w_proj, a_proj);
            break;
        case KernelFunction::Sinc:
            r = image_visibilities(Sinc(s), vis, vis_weights, uvw_lambda, img_pars, w_proj, a_proj);
            break;
        case KernelFunction::Gaussian:
            r = image_visibilities(Gaussian(s), vis, vis_weights, uvw_lambda, img_pars, w_proj, a_proj);
            break;
        case KernelFunction::GaussianSinc:
            r = image_visibilities(GaussianSinc(s), vis, vis_weights, uvw_lambda, img_pars, w_proj, a_proj);
            break;
        case KernelFunction::PSWF:
            r = image_visibilities(PSWF(s), vis, vis_weights, uvw_lambda, img_pars, w_proj, a_proj);
            break;
        default:
            throw std::runtime_error("ImageVisibilities: unknown kernel function");
        }
        vis_grid = std::move(r.first);
        sampling_grid = std::move(r.second);
    }

    arma::Mat<real_t> vis_grid;
    arma::Mat<real_t> sampling_grid;
};

/* stp::IslandParams, src/stp/sourcefind/sourcefind.h:63-133 (fields). */
struct IslandParams {
    int label_idx = 0;
    double extremum_val = 0.0;
    int extremum_y_idx = 0;
    int extremum_x_idx = 0;
    int sign = 0;
    int num_samples = 0;
    BoundingBox bounding_box;
    Gaussian2dParams moments_fit;
    Gaussian2dParams leastsq_fit;
    std::string ceres_report;

    bool operator==(const IslandParams& o) const
    {
        return label_idx == o.label_idx && extremum_val == o.extremum_val && extremum_y_idx == o.extremum_y_idx
            && extremum_x_idx == o.extremum_x_idx && sign == o.sign && num_samples == o.num_samples;
    }
};

/* stp::SourceFindImage, src/stp/sourcefind/sourcefind.h:143-201,
 * sourcefind.cpp:156-292.  Gaussian fitting uses the library's
 * Levenberg-Marquardt fit in place of Ceres (ceres_* are accepted and
 * ignored). */
class SourceFindImage {
public:
    MatStp<int> label_map;
    arma::Col<real_t> label_extrema_val_pos;
    arma::Col<real_t> label_extrema_val_neg;
    arma::uvec label_extrema_linear_idx_pos;
    arma::uvec label_extrema_linear_idx_neg;
    arma::ivec label_extrema_id_pos;
    arma::ivec label_extrema_id_neg;
    arma::mat label_extrema_moments_pos;
    arma::mat label_extrema_moments_neg;
    arma::Col<int> label_extrema_numsamples_pos;
    arma::Col<int> label_extrema_numsamples_neg;
    std::vector<BoundingBox> label_extrema_boundingbox_pos;
    std::vector<BoundingBox> label_extrema_boundingbox_neg;
    double detection_n_sigma;
    double analysis_n_sigma;
    double rms_est;
    real_t bg_level;
    std::vector<IslandParams> islands;
    bool fit_gaussian;

    SourceFindImage() = delete;
    SourceFindImage(
        const arma::Mat<real_t>& input_data,
        double input_detection_n_sigma,
        double input_analysis_n_sigma,
        double input_rms_est = 0.0,
        bool find_negative_sources = true,
        int sigma_clip_iters = 5,
        MedianMethod median_method = MedianMethod::BINAPPROX,
        bool gaussian_fitting = false,
        bool ccl_4connectivity = false,
        bool generate_labelmap = true,
        int source_min_area = 5,
        CeresDiffMethod ceres_diffmethod = CeresDiffMethod::AnalyticDiff_SingleResBlk,
        CeresSolverType ceres_solvertype = CeresSolverType::LinearSearch_LBFGS)
        : detection_n_sigma(input_detection_n_sigma)
        , analysis_n_sigma(input_analysis_n_sigma)
        , rms_est(input_rms_est)
        , bg_level(0)
        , fit_gaussian(gaussian_fitting)
    {
        using namespace stpgpu_detail;
        (void)ceres_diffmethod;
        (void)ceres_solvertype;
        stpgpu_sf_pars p {};
        p.detection_n_sigma = input_detection_n_sigma;
        p.analysis_n_sigma = input_analysis_n_sigma;
        p.rms_est = input_rms_est;
        p.find_negative_sources = find_negative_sources ? 1 : 0;
        p.sigma_clip_iters = sigma_clip_iters;
        p.median_method = int32_t(median_method);
        p.gaussian_fitting = gaussian_fitting ? 1 : 0;
        p.ccl_4connectivity = ccl_4connectivity ? 1 : 0;
        p.generate_labelmap = generate_labelmap ? 1 : 0;
        p.source_min_area = source_min_area;
        p.ccl_slice_cols = 0;
        const int rows = int(input_data.n_rows), cols = int(input_data.n_cols);
        label_map.set_size(rows, cols);
        stpgpu_context* c = context();
        std::vector<stpgpu_island> found(4096);
        int32_t n = 0;
        stpgpu_sf_info info {};
        for (;;) {
            const stpgpu_status s = stpgpu_source_find_ex(c, input_data.memptr(), single ? STPGPU_F32 : STPGPU_F64,
                rows, cols, &p, label_map.memptr(), 0, found.data(), int32_t(found.size()), &n, &info);
            if (s == STPGPU_ERR_CAPACITY && size_t(n) > found.size()) {
                found.resize(size_t(n));
                continue;
            }
            check(c, s);
            break;
        }
        bg_level = real_t(info.bg_level);
        rms_est = info.rms_est;
        islands.resize(size_t(n));
        for (int32_t k = 0; k < n; k++) {
            const stpgpu_island& f = found[size_t(k)];
            IslandParams& d = islands[size_t(k)];
            d.label_idx = f.label_idx;
            d.extremum_val = f.extremum_val;
            d.extremum_y_idx = f.extremum_y_idx;
            d.extremum_x_idx = f.extremum_x_idx;
            d.sign = f.sign;
            d.num_samples = f.num_samples;
            d.bounding_box.top = f.bbox_top;
            d.bounding_box.bottom = f.bbox_bottom;
            d.bounding_box.left = f.bbox_left;
            d.bounding_box.right = f.bbox_right;
            const double* m = f.moments_fit;
            d.moments_fit.amplitude = m[0];
            d.moments_fit.x_centre = m[1];
            d.moments_fit.y_centre = m[2];
            d.moments_fit.semimajor = m[3];
            d.moments_fit.semiminor = m[4];
            d.moments_fit.theta = m[5];
            const double* q = f.leastsq_fit;
            d.leastsq_fit.amplitude = q[0];
            d.leastsq_fit.x_centre = q[1];
            d.leastsq_fit.y_centre = q[2];
            d.leastsq_fit.semimajor = q[3];
            d.leastsq_fit.semiminor = q[4];
            d.leastsq_fit.theta = q[5];
            if (f.fit_iterations > 0)
                d.ceres_report = "Levenberg-Marquardt iterations: " + std::to_string(f.fit_iterations);
        }
    }
};

} // namespace stp

#endif /* STPGPU_STP_HPP */
