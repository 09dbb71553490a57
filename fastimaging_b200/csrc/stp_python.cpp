// pybind11 module `stp_python`: the reference's Python binding
// (src/stp-python/stp_python.cpp:17-284, src/stp-python/stp_python.h) with the
// same function names, argument names, defaults, enum names and return
// values, running the B200 imager and source finder through the C ABI
// (include/stpgpu.h).  Arrays are coerced to F-order float64 / complex128 as
// the reference's forcecast array types do (stp_python.h:17-20), outputs are
// new F-order numpy arrays, and errors raise RuntimeError.
//
// One library context per device, created on first use (device from the
// STPGPU_DEVICE environment variable, default 0); calls on it are serialised
// by a mutex, the GIL is released while the GPU works.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <complex>
#include <cstdlib>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "stpgpu.h"

namespace py = pybind11;

namespace {

using np_complex_double_array = py::array_t<std::complex<double>, py::array::f_style | py::array::forcecast>;
using np_double_array = py::array_t<double, py::array::f_style | py::array::forcecast>;

// Enumerations with the reference's names and values (src/stp/types.h).
enum class KernelFunction { TopHat = 0, Triangle, Sinc, Gaussian, GaussianSinc, PSWF };
enum class FFTRoutine { FFTW_ESTIMATE_FFT = 0, FFTW_MEASURE_FFT, FFTW_PATIENT_FFT, FFTW_WISDOM_FFT, FFTW_WISDOM_INPLACE_FFT };
enum class InterpType { LINEAR = 0, CUBIC = 1, COSINE = 2 }; // stp::InterpType, src/stp/types.h:55-59
enum class MedianMethod { ZEROMEDIAN = 0, BINMEDIAN, BINAPPROX, NTHELEMENT };
enum class CeresDiffMethod { AutoDiff = 0, AutoDiff_SingleResBlk, AnalyticDiff, AnalyticDiff_SingleResBlk };
enum class CeresSolverType { LinearSearch_BFGS = 0, LinearSearch_LBFGS, TrustRegion_DenseQR };

// stp::Gaussian2dParams (src/stp/sourcefind/fitting.h:90-110): all zero by default.
struct Gaussian2dParams {
    double amplitude = 0.0, x_centre = 0.0, y_centre = 0.0, semimajor = 0.0, semiminor = 0.0, theta = 0.0;
};

struct Session {
    std::mutex mu;
    stpgpu_context* ctx = nullptr;
};

Session& session()
{
    static Session s;
    return s;
}

stpgpu_context* context_locked(Session& s)
{
    if (!s.ctx) {
        const char* e = std::getenv("STPGPU_DEVICE");
        const int dev = e ? std::atoi(e) : 0;
        stpgpu_context* c = nullptr;
        const stpgpu_status st = stpgpu_create(dev, &c);
        if (st != STPGPU_OK)
            throw std::runtime_error("stp_python: cannot create a GPU context on device " + std::to_string(dev)
                + " (status " + std::to_string(int(st)) + ")");
        s.ctx = c;
    }
    return s.ctx;
}

void check(stpgpu_context* c, stpgpu_status st)
{
    if (st != STPGPU_OK)
        throw std::runtime_error(std::string("stp_python: ") + stpgpu_last_error(c));
}

py::array_t<double, py::array::f_style> f_matrix(py::ssize_t rows, py::ssize_t cols)
{
    return py::array_t<double, py::array::f_style>({ rows, cols });
}

py::tuple image_visibilities_wrapper(np_complex_double_array vis, np_double_array snr_weights,
    np_double_array uvw_lambda, unsigned image_size, double cell_size, double padding_factor,
    KernelFunction kernel_func, unsigned kernel_support, bool kernel_exact, unsigned oversampling, bool generate_beam,
    bool gridding_correction, bool analytic_gcf, FFTRoutine r_fft, std::string fft_wisdom_filename,
    unsigned num_wplanes, bool wplanes_median, unsigned max_wpconv_support, bool hankel_opt, bool hankel_proj_slice,
    unsigned undersampling_opt, double kernel_trunc_perc, InterpType interp_type, unsigned aproj_numtimesteps,
    double obs_dec, double obs_ra, bool aproj_opt, double aproj_mask_perc, np_double_array lha,
    np_double_array pbeam_coefs)
{
    (void)fft_wisdom_filename;
    if (uvw_lambda.ndim() != 2 || uvw_lambda.shape(1) != 3)
        throw std::runtime_error("stp_python: uvw_lambda must have shape (n_vis, 3)");
    const int64_t n = int64_t(uvw_lambda.shape(0));
    if (int64_t(vis.size()) < n || int64_t(snr_weights.size()) < n)
        throw std::runtime_error("stp_python: vis and snr_weights need n_vis entries");
    if (aproj_numtimesteps > 0 && int64_t(lha.size()) < n)
        throw std::runtime_error("stp_python: lha needs n_vis entries");

    // image sizes rounded up to multiples of 4 (stp_python.cpp:60-67)
    while (image_size % 4)
        image_size++;
    unsigned padded = unsigned(double(image_size) * padding_factor);
    while (padded % 4)
        padded++;

    stpgpu_imager_pars ip {};
    ip.image_size = int32_t(image_size);
    ip.padded_image_size = int32_t(padded);
    ip.cell_size = cell_size;
    ip.padding_factor = padding_factor;
    ip.kernel_function = int32_t(kernel_func);
    ip.kernel_support = int32_t(kernel_support);
    ip.kernel_exact = kernel_exact;
    ip.oversampling = int32_t(oversampling);
    ip.generate_beam = generate_beam;
    ip.gridding_correction = gridding_correction;
    ip.analytic_gcf = analytic_gcf;
    ip.r_fft = int32_t(r_fft);
    stpgpu_wproj_pars wp {};
    wp.num_wplanes = int32_t(num_wplanes);
    wp.max_wpconv_support = int32_t(max_wpconv_support);
    wp.undersampling_opt = int32_t(undersampling_opt);
    wp.kernel_trunc_perc = kernel_trunc_perc;
    wp.hankel_opt = hankel_opt;
    wp.hankel_proj_slice = hankel_proj_slice;
    wp.interp_type = int32_t(interp_type);
    wp.wplanes_median = wplanes_median;
    stpgpu_aproj_pars ap {};
    ap.num_timesteps = int32_t(aproj_numtimesteps);
    ap.obs_dec = obs_dec;
    ap.obs_ra = obs_ra;
    ap.aproj_opt = aproj_opt;
    ap.aproj_mask_perc = aproj_mask_perc;
    ap.lha = aproj_numtimesteps > 0 ? lha.data() : nullptr;
    ap.pbeam_coefs = pbeam_coefs.size() ? pbeam_coefs.data() : nullptr;
    ap.n_pbeam_coefs = int32_t(pbeam_coefs.size());

    auto image = f_matrix(image_size, image_size);
    auto beam = f_matrix(generate_beam ? image_size : 0, generate_beam ? image_size : 0);
    const double* pv = reinterpret_cast<const double*>(vis.data());
    const double* pw = snr_weights.data();
    const double* puvw = uvw_lambda.data();
    double* pi = image.mutable_data();
    double* pb = generate_beam ? beam.mutable_data() : nullptr;
    stpgpu_imager_info info {};
    Session& s = session();
    {
        py::gil_scoped_release nogil;
        std::lock_guard<std::mutex> lk(s.mu);
        stpgpu_context* c = context_locked(s);
        check(c, stpgpu_image_visibilities(c, pv, pw, puvw, n, &ip, &wp, &ap, pi, pb, &info));
    }
    py::tuple result(2);
    if (info.image_size == 0) {
        // zero sampling total: the reference returns empty matrices (imager.h:355)
        result[0] = f_matrix(0, 0);
        result[1] = f_matrix(0, 0);
        return result;
    }
    result[0] = image;
    result[1] = beam;
    return result;
}

std::vector<std::tuple<int, double, int, int, int, Gaussian2dParams, Gaussian2dParams, std::string>>
source_find_wrapper(np_double_array image_data, double detection_n_sigma, double analysis_n_sigma, double rms_est,
    bool find_negative_sources, unsigned sigma_clip_iters, MedianMethod median_method, bool gaussian_fitting,
    bool ccl_4connectivity, bool generate_labelmap, int source_min_area, CeresDiffMethod ceres_diffmethod,
    CeresSolverType ceres_solvertype)
{
    (void)ceres_diffmethod;
    (void)ceres_solvertype;
    if (image_data.ndim() != 2)
        throw std::runtime_error("stp_python: image_data must be 2-D");
    const int32_t rows = int32_t(image_data.shape(0)), cols = int32_t(image_data.shape(1));
    stpgpu_sf_pars p {};
    p.detection_n_sigma = detection_n_sigma;
    p.analysis_n_sigma = analysis_n_sigma;
    p.rms_est = rms_est;
    p.find_negative_sources = find_negative_sources;
    p.sigma_clip_iters = int32_t(sigma_clip_iters);
    p.median_method = int32_t(median_method);
    p.gaussian_fitting = gaussian_fitting;
    p.ccl_4connectivity = ccl_4connectivity;
    p.generate_labelmap = generate_labelmap;
    p.source_min_area = source_min_area;
    p.ccl_slice_cols = 0;
    const double* img = image_data.data();
    std::vector<stpgpu_island> isl(1024);
    int32_t nis = 0;
    Session& s = session();
    {
        py::gil_scoped_release nogil;
        std::lock_guard<std::mutex> lk(s.mu);
        stpgpu_context* c = context_locked(s);
        for (;;) {
            stpgpu_sf_info info {};
            const stpgpu_status st = stpgpu_source_find(c, img, rows, cols, &p, nullptr, isl.data(),
                int32_t(isl.size()), &nis, &info);
            if (st == STPGPU_ERR_CAPACITY && nis > int32_t(isl.size())) {
                isl.resize(size_t(nis));
                continue;
            }
            check(c, st);
            break;
        }
    }
    std::vector<std::tuple<int, double, int, int, int, Gaussian2dParams, Gaussian2dParams, std::string>> out;
    out.reserve(size_t(nis));
    for (int32_t i = 0; i < nis; i++) {
        const stpgpu_island& r = isl[size_t(i)];
        Gaussian2dParams m, l;
        m.amplitude = r.moments_fit[0];
        m.x_centre = r.moments_fit[1];
        m.y_centre = r.moments_fit[2];
        m.semimajor = r.moments_fit[3];
        m.semiminor = r.moments_fit[4];
        m.theta = r.moments_fit[5];
        l.amplitude = r.leastsq_fit[0];
        l.x_centre = r.leastsq_fit[1];
        l.y_centre = r.leastsq_fit[2];
        l.semimajor = r.leastsq_fit[3];
        l.semiminor = r.leastsq_fit[4];
        l.theta = r.leastsq_fit[5];
        std::string report;
        if (gaussian_fitting)
            report = r.num_samples < 3 ? "least-squares fit not run: source of one or two pixels"
                                       : "Levenberg-Marquardt fit, " + std::to_string(r.fit_iterations) + " iterations";
        out.emplace_back(r.sign, r.extremum_val, r.extremum_x_idx, r.extremum_y_idx, r.num_samples, m, l, report);
    }
    return out;
}

} // namespace

PYBIND11_MODULE(stp_python, m)
{
    m.doc() = "The Slow Transients Pipeline (B200 imager and source finder)";

    py::enum_<KernelFunction>(m, "KernelFunction")
        .value("TopHat", KernelFunction::TopHat)
        .value("Triangle", KernelFunction::Triangle)
        .value("Sinc", KernelFunction::Sinc)
        .value("Gaussian", KernelFunction::Gaussian)
        .value("GaussianSinc", KernelFunction::GaussianSinc)
        .value("PSWF", KernelFunction::PSWF);
    py::enum_<FFTRoutine>(m, "FFTRoutine")
        .value("FFTW_ESTIMATE_FFT", FFTRoutine::FFTW_ESTIMATE_FFT)
        .value("FFTW_MEASURE_FFT", FFTRoutine::FFTW_MEASURE_FFT)
        .value("FFTW_PATIENT_FFT", FFTRoutine::FFTW_PATIENT_FFT)
        .value("FFTW_WISDOM_FFT", FFTRoutine::FFTW_WISDOM_FFT)
        .value("FFTW_WISDOM_INPLACE_FFT", FFTRoutine::FFTW_WISDOM_INPLACE_FFT);
    py::enum_<InterpType>(m, "InterpType")
        .value("LINEAR", InterpType::LINEAR)
        .value("COSINE", InterpType::COSINE)
        .value("CUBIC", InterpType::CUBIC);
    py::enum_<MedianMethod>(m, "MedianMethod")
        .value("ZEROMEDIAN", MedianMethod::ZEROMEDIAN)
        .value("BINMEDIAN", MedianMethod::BINMEDIAN)
        .value("BINAPPROX", MedianMethod::BINAPPROX)
        .value("NTHELEMENT", MedianMethod::NTHELEMENT);
    py::enum_<CeresDiffMethod>(m, "CeresDiffMethod")
        .value("AutoDiff", CeresDiffMethod::AutoDiff)
        .value("AutoDiff_SingleResBlk", CeresDiffMethod::AutoDiff_SingleResBlk)
        .value("AnalyticDiff", CeresDiffMethod::AnalyticDiff)
        .value("AnalyticDiff_SingleResBlk", CeresDiffMethod::AnalyticDiff_SingleResBlk);
    py::enum_<CeresSolverType>(m, "CeresSolverType")
        .value("LinearSearch_BFGS", CeresSolverType::LinearSearch_BFGS)
        .value("LinearSearch_LBFGS", CeresSolverType::LinearSearch_LBFGS)
        .value("TrustRegion_DenseQR", CeresSolverType::TrustRegion_DenseQR);

    py::class_<Gaussian2dParams>(m, "Gaussian2dParams")
        .def(py::init<>())
        .def_readwrite("amplitude", &Gaussian2dParams::amplitude)
        .def_readwrite("x_centre", &Gaussian2dParams::x_centre)
        .def_readwrite("y_centre", &Gaussian2dParams::y_centre)
        .def_readwrite("semimajor", &Gaussian2dParams::semimajor)
        .def_readwrite("semiminor", &Gaussian2dParams::semiminor)
        .def_readwrite("theta", &Gaussian2dParams::theta)
        .def("__repr__", [](const Gaussian2dParams& g) {
            return "Gaussian2dParams=[" + std::to_string(g.amplitude) + ", " + std::to_string(g.x_centre) + ", "
                + std::to_string(g.y_centre) + ", " + std::to_string(g.semimajor) + ", "
                + std::to_string(g.semiminor) + ", " + std::to_string(g.theta) + "]";
        });

    m.def("image_visibilities_wrapper", &image_visibilities_wrapper, "Compute image visibilities (gridding + ifft).",
        py::arg("vis"), py::arg("snr_weights"), py::arg("uvw_lambda"), py::arg("image_size"), py::arg("cell_size"),
        py::arg("padding_factor") = 1.0, py::arg("kernel_func") = KernelFunction::PSWF,
        py::arg("kernel_support") = 3, py::arg("kernel_exact") = true, py::arg("kernel_oversampling") = 8,
        py::arg("generate_beam") = false, py::arg("gridding_correction") = true, py::arg("analytic_gcf") = false,
        py::arg("r_fft") = FFTRoutine::FFTW_ESTIMATE_FFT, py::arg("fft_wisdom_filename") = std::string(),
        py::arg("num_wplanes") = 0, py::arg("wplanes_median") = false, py::arg("max_wpconv_support") = 0,
        py::arg("hankel_opt") = false, py::arg("hankel_proj_slice") = false, py::arg("undersampling_opt") = 1,
        py::arg("kernel_trunc_perc") = 0.0, py::arg("interp_type") = InterpType::LINEAR,
        py::arg("aproj_numtimesteps") = 0, py::arg("obs_dec") = 0.0, py::arg("obs_ra") = 0.0,
        py::arg("aproj_opt") = false, py::arg("aproj_mask_perc") = 0.0, py::arg("lha") = np_double_array(),
        py::arg("pbeam_coefs") = np_double_array());

    m.def("source_find_wrapper", &source_find_wrapper,
        "Find connected regions which peak above/below a given threshold.", py::arg("image_data"),
        py::arg("detection_n_sigma"), py::arg("analysis_n_sigma"), py::arg("rms_est") = 0.0,
        py::arg("find_negative_sources") = true, py::arg("sigma_clip_iters") = 5,
        py::arg("median_method") = MedianMethod::BINAPPROX, py::arg("gaussian_fitting") = false,
        py::arg("ccl_4connectivity") = false, py::arg("generate_labelmap") = true, py::arg("source_min_area") = 5,
        py::arg("ceres_diffmethod") = CeresDiffMethod::AutoDiff_SingleResBlk,
        py::arg("ceres_solvertype") = CeresSolverType::LinearSearch_BFGS);
}
