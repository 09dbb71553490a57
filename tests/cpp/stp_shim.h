// Test scaffolding for the C++ adapter: the reference's public parameter
// types, enums and functor class names (src/stp/types.h:20-316,
// src/stp/convolution/conv_func.h functor classes, src/stp/sourcefind/fitting.h
// BoundingBox / Gaussian2dParams, src/stp/common/matstp.h MatStp) declared with
// the same names, fields and defaults, so that a translation unit written
// against the reference's headers compiles here against the adapter.  The
// functor classes carry no arithmetic: the adapter identifies them by type.
#pragma once

#include <string>
#include <vector>

#include "arma_shim.h"

#ifdef USE_FLOAT
using real_t = float;
#else
using real_t = double;
#endif

namespace stp {

enum struct KernelFunction { TopHat, Triangle, Sinc, Gaussian, GaussianSinc, PSWF };
enum struct FFTRoutine { FFTW_ESTIMATE_FFT, FFTW_MEASURE_FFT, FFTW_PATIENT_FFT, FFTW_WISDOM_FFT, FFTW_WISDOM_INPLACE_FFT };
enum struct InterpType { LINEAR, CUBIC, COSINE };
enum struct MedianMethod { ZEROMEDIAN, BINMEDIAN, BINAPPROX, NTHELEMENT };
enum struct CeresDiffMethod { AutoDiff, AutoDiff_SingleResBlk, AnalyticDiff, AnalyticDiff_SingleResBlk };
enum struct CeresSolverType { LinearSearch_BFGS, LinearSearch_LBFGS, TrustRegion_DenseQR };

struct ImagerPars {
    ImagerPars() = default;
    ImagerPars(unsigned size, double cell, double padding = 1.0, KernelFunction kf = KernelFunction::PSWF,
        unsigned support = 3, bool exact = true, unsigned os = 1, bool beam = false, bool correction = true,
        bool analytic = true)
        : image_size(size), cell_size(cell), padding_factor(padding), kernel_function(kf), kernel_support(support),
          kernel_exact(exact), oversampling(os), generate_beam(beam), gridding_correction(correction),
          analytic_gcf(analytic)
    {
        padded_image_size = unsigned(image_size * padding_factor);
    }
    unsigned image_size = 0;
    unsigned padded_image_size = 0;
    double cell_size = 0.0;
    double padding_factor = 1.0;
    KernelFunction kernel_function = KernelFunction::PSWF;
    unsigned kernel_support = 0;
    bool kernel_exact = true;
    unsigned oversampling = 0;
    bool generate_beam = false;
    bool gridding_correction = false;
    bool analytic_gcf = false;
    FFTRoutine r_fft = FFTRoutine::FFTW_ESTIMATE_FFT;
    std::string fft_wisdom_filename;
};

struct W_ProjectionPars {
    unsigned num_wplanes = 0;
    unsigned max_wpconv_support = 0;
    unsigned undersampling_opt = 1;
    double kernel_trunc_perc = 0.0;
    bool hankel_opt = false;
    bool hankel_proj_slice = false;
    InterpType interp_type = InterpType::LINEAR;
    bool wplanes_median = false;
};

struct A_ProjectionPars {
    unsigned num_timesteps = 0;
    double obs_dec = 0.0;
    double obs_ra = 0.0;
    bool aproj_opt = false;
    double aproj_mask_perc = 0.0;
    arma::mat lha;
    std::vector<double> pbeam_coefs;
};

class TopHat {
public:
    explicit TopHat(double) { }
};
class Triangle {
public:
    explicit Triangle(double) { }
};
class Sinc {
public:
    explicit Sinc(double = 0.0, double = 1.0) { }
};
class Gaussian {
public:
    explicit Gaussian(double = 0.0, double = 1.0) { }
};
class GaussianSinc {
public:
    explicit GaussianSinc(double = 0.0, double = 2.52, double = 1.55) { }
};
class PSWF {
public:
    explicit PSWF(double = 0.0) { }
};

struct BoundingBox {
    int top = 0, bottom = 0, left = 0, right = 0;
};

struct Gaussian2dParams {
    double amplitude = 0.0, x_centre = 0.0, y_centre = 0.0, semimajor = 0.0, semiminor = 0.0, theta = 0.0;
};

template <typename T>
class MatStp : public arma::Mat<T> {
};

} // namespace stp
