// tomogpi_exe -- command-line drop-in for TomoGPI_exe's --op=proj / --op=back / gradient
// paths (src/TomoGPI_exe/TomoGPI_exe.cu:152-377, src/TomoGPI_lib/src/CPP/Iter3D_main.cu:14-421).
//
//   tomogpi_exe <N> [--pair=RSVI|SiddonVI|SIDDONVI] [--op=proj|back|back_fdk|laplacien|reg_GG|tiff5|tiff4]
//               [--compute=CUDA|CPU|C]
//               [--storage=mem_CPU|mem_GPU] [--precision=float] [--ngpu=1] [--nstreams=k]
//               [--no_load] [--no_save] [--workdir=DIR] [--sino=FILE] [--volume=FILE]
//
// Reads Projections_<N>/configCT, configIteration and configComputeArchitecture (first
// token match per field, Config.cpp:35-69); command-line switches override the file. Files
// go where the reference puts them (Iter3D_main.cu:54-336): outputs of the operator ops in
// the current directory, the measured sinogram read from <workdir>/<tiffName>.s (configTiff;
// <workdir>/proj.s without one; --sino overrides).
// --op=proj: projects realVolumeName (or --volume) and writes proj.s; --op=back:
// backprojects the measured sinogram and writes back.v; --op=back_fdk: the
// FDK-weighted backprojection of that sinogram (Iter3D_main.cu:296-316; the reference
// expects it already ramp-filtered, --ramp_filter filters it first) into back_fdk.v; without --op: runs
// gradientIterationNb iterations of the simple gradient and writes
// <workdir>TomoIter/Results/Result_<date>/finalVolume.v;
// --op=tiff5|tiff4: builds the negative-log sinogram <tiffName>.s from the detector files
// named in configTiff (<workdir>/../tif, <workdir>/../Calibration), on the host;
// --op=laplacien / --op=reg_GG: the Laplacian / regulariser gradient of realVolumeName into
// laplacien.v / GG.v.
// Prints "Time computation : <ms> ms" like the reference.
// Quirks kept from the reference: --storage=mem_GPU always uses the RSVI mem_GPU pair
// (TomoGPI_exe.cu:343-347). Accepted spellings: --pair=SiddonVI (reference) and
// SIDDONVI (its README); --compute=CPU (reference) and C (README). All compute runs in
// libtomogpi_b200 on the GPU; OCL/FPGA targets are rejected.
#include <chrono>
#include <ctime>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <initializer_list>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "tomogpi_b200.h"

namespace {

std::string read_field(const std::string& path, const std::string& name, bool required = true,
                       const std::string& dflt = "") {
    std::ifstream f(path);
    if (!f) {
        if (!required) return dflt;
        std::cerr << "Unable to open file " << path << std::endl;
        std::exit(EXIT_FAILURE);
    }
    std::string row;
    while (std::getline(f, row)) {
        std::istringstream ss(row);
        std::string tok;
        while (ss >> tok) {
            if (tok == name) {
                std::string v;
                ss >> v;
                return v;
            }
        }
    }
    if (!required) return dflt;
    std::cerr << "Unable to find field " << name << " in " << path << std::endl;
    std::exit(EXIT_FAILURE);
}

bool flag(int argc, char** argv, const char* name, std::string* value) {
    const size_t n = std::strlen(name);
    for (int i = 2; i < argc; ++i) {
        const char* a = argv[i];
        while (*a == '-') ++a;
        if (std::strncmp(a, name, n) == 0 && (a[n] == '=' || a[n] == 0)) {
            if (value) *value = a[n] == '=' ? std::string(a + n + 1) : std::string();
            return true;
        }
    }
    return false;
}

template <typename T>
bool load_raw(const std::string& path, std::vector<T>& v) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * v.size());
    return (size_t)f.gcount() == sizeof(T) * v.size();
}

// Raw values as the reference writes them (Sinogram3D.cu:138-184, Volume.cu:248-272), plus
// a text sidecar <path>.hdr: "dtype <f4>" and "shape <slowest> ... <fastest>".
void save_raw(const std::string& path, const std::vector<float>& v, std::initializer_list<long> shape) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), sizeof(float) * v.size());
    std::ofstream h(path + ".hdr");
    h << "dtype <f4\nshape";
    for (long d : shape) h << ' ' << d;
    h << '\n';
}

void die(tomo_status s, const char* what) {
    if (s != TOMO_OK) {
        std::cerr << what << " failed: " << tomo_last_error() << std::endl;
        std::exit(EXIT_FAILURE);
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::printf("usage: tomogpi_exe <N> [--pair=...] [--op=proj|back] ...\n");
        return -1;
    }
    std::string wd = "Projections_" + std::to_string(std::strtoul(argv[1], nullptr, 10)) + "/";
    std::string v;
    if (flag(argc, argv, "workdir", &v)) wd = v.back() == '/' ? v : v + "/";
    const std::string ct = wd + "configCT", it = wd + "configIteration", ca = wd + "configComputeArchitecture";

    // switches: file values, overridden by the command line (TomoGPI_exe.cu:200-273)
    std::string pair = read_field(ca, "pair", false, "PAIR_RSVI");
    std::string storage = read_field(ca, "storage", false, "mem_CPU");
    std::string compute = read_field(ca, "compute", false, "COMPUTE_CUDA");
    std::string precision = read_field(ca, "precision", false, "float");
    if (flag(argc, argv, "pair", &v)) pair = v;
    if (flag(argc, argv, "storage", &v)) storage = v;
    if (flag(argc, argv, "compute", &v)) compute = v;
    if (flag(argc, argv, "precision", &v)) precision = v;
    const bool siddon = pair == "SiddonVI" || pair == "SIDDONVI" || pair == "PAIR_SIDDONVI";
    const bool mem_gpu = storage == "mem_GPU";
    if (precision != "float") {
        std::cerr << "precision " << precision << " not supported (float only)" << std::endl;
        return EXIT_FAILURE;
    }
    if (compute == "OCL" || compute == "GPU_FPGA" || compute == "COMPUTE_OCL") {
        std::cerr << "compute target " << compute << " (OpenCL/FPGA) is not available" << std::endl;
        return EXIT_FAILURE;
    }
    if (mem_gpu && siddon) std::cout << "\tmem_GPU uses the RSVI pair (as TomoGPI_exe does)" << std::endl;
    // TomoGPI_exe's mem_MGPU branches are empty (TomoGPI_exe.cu:295, 349, 371): it runs nothing.
    // Here it runs as mem_CPU on one GPU; one job over several GPUs is tomogpi_b200.sharded.
    if (storage == "mem_MGPU") std::cout << "\tmem_MGPU runs as mem_CPU on one GPU" << std::endl;
    const tomo_projector P = mem_gpu ? TOMO_PROJ_RS_UM : (siddon ? TOMO_PROJ_SIDDON_REF : TOMO_PROJ_RS);
    const tomo_backprojector B = mem_gpu ? TOMO_BACK_VI_UM : TOMO_BACK_VI;

    tomo_config_ct c{};
    c.fod = std::atof(read_field(ct, "FOD").c_str());
    c.fdd = std::atof(read_field(ct, "FDD").c_str());
    c.projection_nb = std::atoi(read_field(ct, "projectionNb").c_str());
    c.num_start_angle = std::atof(read_field(ct, "numStartAngle").c_str());
    c.den_start_angle = std::atof(read_field(ct, "denStartAngle").c_str());
    c.num_stop_angle = std::atof(read_field(ct, "numStopAngle").c_str());
    c.den_stop_angle = std::atof(read_field(ct, "denStopAngle").c_str());
    c.u_detector_size = (float)std::atof(read_field(ct, "horizontalDetectorSize").c_str());
    c.v_detector_size = (float)std::atof(read_field(ct, "verticalDetectorSize").c_str());
    c.u_detector_pixel_nb = std::atoi(read_field(ct, "horizontalDetectorPixelNb").c_str());
    c.v_detector_pixel_nb = std::atoi(read_field(ct, "verticalDetectorPixelNb").c_str());
    c.x_volume_size = (float)std::atof(read_field(ct, "xVolumeSize").c_str());
    c.y_volume_size = (float)std::atof(read_field(ct, "yVolumeSize").c_str());
    c.z_volume_size = (float)std::atof(read_field(ct, "zVolumeSize").c_str());
    c.x_volume_pixel_nb = std::atoi(read_field(ct, "xVolumePixelNb").c_str());
    c.y_volume_pixel_nb = std::atoi(read_field(ct, "yVolumePixelNb").c_str());
    c.z_volume_pixel_nb = std::atoi(read_field(ct, "zVolumePixelNb").c_str());
    const size_t nvox = (size_t)c.x_volume_pixel_nb * c.y_volume_pixel_nb * c.z_volume_pixel_nb;
    const size_t nsino = (size_t)c.u_detector_pixel_nb * c.v_detector_pixel_nb * c.projection_nb;
    const bool no_save = flag(argc, argv, "no_save", nullptr);
    const bool no_load = flag(argc, argv, "no_load", nullptr);

    std::string op;
    flag(argc, argv, "op", &op);
    // The measured sinogram: <workdir>/<tiffName>.s (Iter3D.cu:27-30, tiffName from configTiff);
    // without a configTiff, <workdir>/proj.s. --sino overrides either.
    auto measured_sinogram = [&]() {
        std::string name = read_field(wd + "configTiff", "tiffName", false, "");
        std::string path = name.empty() ? wd + "proj.s" : wd + "/" + name + ".s";
        if (flag(argc, argv, "sino", &v)) path = v;
        return path;
    };
    if (op == "tiff5" || op == "tiff4") {
        // detector files -> normalised negative-log sinogram <workdir>/<tiffName>.s
        // (Iter3D_main.cu:317-336, Iter3D.cu:27-30); host only, no device needed
        const std::string tf = wd + "configTiff";
        auto num = [&](const char* name) { return std::atoi(read_field(tf, name).c_str()); };
        tomo_tiff_config t{};
        t.total_projection_nb = num("totalProjectionNb");
        t.used_projection_nb = num("usedProjectionNb");
        t.u_initial_nb = num("uDetectorPixelInitialNb");
        t.v_initial_nb = num("vDetectorPixelInitialNb");
        t.u_final_nb = num("uDetectorPixelFinalNb");
        t.v_final_nb = num("vDetectorPixelFinalNb");
        t.u_center_final = num("uDetectorCenterFinal");
        t.v_center_final = num("vDetectorCenterFinal");
        t.u_calibration_nb = num("uCalibrationImagePixelNb");
        t.v_calibration_nb = num("vCalibrationImagePixelNb");
        t.calibration_energy_nb = num("CalibrationEnergyNb");
        t.digits = op == "tiff5" ? 5 : 4;
        const std::string name = read_field(tf, "tiffName");
        const std::string calib = wd + "../Calibration/" + read_field(tf, "calibrationTiffName");
        std::vector<float> sino((size_t)t.u_final_nb * t.v_final_nb * (t.used_projection_nb > 0 ? t.used_projection_nb : 0));
        const auto t0 = std::chrono::high_resolution_clock::now();
        die(tomo_tiff_negative_log_sinogram(&t, (wd + "../tif").c_str(), name.c_str(), calib.c_str(), sino.data()),
            "tomo_tiff_negative_log_sinogram");
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
        std::cout << "createNormalizedMeanNegativeLogSinogram done" << std::endl;
        save_raw(wd + name + ".s", sino, {t.used_projection_nb, t.v_final_nb, t.u_final_nb});
        std::cout << "Real sinogram from tiff created" << std::endl;
        std::cout << "Time computation : " << ms << " ms" << std::endl;
        return 0;
    }
    tomo_context* ctx = nullptr;
    die(tomo_context_create(&c, 0, &ctx), "tomo_context_create");
    using clk = std::chrono::high_resolution_clock;
    double ms = 0.0;
    if (op == "proj") {
        std::vector<float> vol(nvox, 0.f), sino(nsino, 0.f);
        std::string name = read_field(ct, "realVolumeName", false, "none");
        if (flag(argc, argv, "volume", &v)) name = v;
        if (!no_load) {
            if (name == "none" || !load_raw(name, vol)) {
                std::cerr << "cannot load the volume to project (" << name << ")" << std::endl;
                return EXIT_FAILURE;
            }
        }
        auto t0 = clk::now();
        die(tomo_project_host(ctx, P, vol.data(), sino.data()), "doProjection");
        ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        if (!no_save) save_raw("proj.s", sino, {c.projection_nb, c.v_detector_pixel_nb, c.u_detector_pixel_nb});
    } else if (op == "back") {
        std::vector<float> vol(nvox, 0.f), sino(nsino, 0.f);
        const std::string name = measured_sinogram();
        if (!no_load && !load_raw(name, sino)) {
            std::cerr << "cannot load the sinogram " << name << std::endl;
            return EXIT_FAILURE;
        }
        auto t0 = clk::now();
        die(tomo_backproject_host(ctx, B, sino.data(), vol.data()), "doBackProjection");
        ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        if (!no_save) save_raw("back.v", vol, {c.z_volume_pixel_nb, c.y_volume_pixel_nb, c.x_volume_pixel_nb});
    } else if (op == "back_fdk") {
        std::vector<float> vol(nvox, 0.f), sino(nsino, 0.f);
        const std::string name = measured_sinogram();
        if (!no_load && !load_raw(name, sino)) {
            std::cerr << "cannot load the sinogram " << name << std::endl;
            return EXIT_FAILURE;
        }
        const bool ramp = flag(argc, argv, "ramp_filter", nullptr);
        auto t0 = clk::now();
        if (ramp) die(tomo_ramp_filter_host(ctx, sino.data(), sino.data(), 16, 1.0), "ramp filter");
        die(tomo_backproject_host(ctx, TOMO_BACK_FDK, sino.data(), vol.data()), "doBackProjection (fdk)");
        ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        if (!no_save) save_raw("back_fdk.v", vol, {c.z_volume_pixel_nb, c.y_volume_pixel_nb, c.x_volume_pixel_nb});
    } else if (op == "laplacien" || op == "reg_GG") {
        // Iter3D_main.cu:215-272: the {-1,2,-1} Laplacian of realVolumeName (laplacien.v), or
        // the regulariser criterion applied twice to dJ = 0 as the reference's timing loop
        // does (GG.v; the Huber criterion under penaltyFunction Huber)
        std::vector<float> vol(nvox, 0.f), out(nvox, 0.f);
        std::string name = read_field(ct, "realVolumeName", false, "none");
        if (flag(argc, argv, "volume", &v)) name = v;
        if (!no_load && (name == "none" || !load_raw(name, vol))) {
            std::cerr << "cannot load the volume (" << name << ")" << std::endl;
            return EXIT_FAILURE;
        }
        auto t0 = clk::now();
        if (op == "laplacien") {
            die(tomo_laplacian_host(0, vol.data(), out.data(), c.x_volume_pixel_nb, c.y_volume_pixel_nb,
                                    c.z_volume_pixel_nb),
                "doSeparableConvolution3D");
        } else {
            const bool huber = read_field(it, "penaltyFunction", false, "GGaussian") == "Huber";
            const double lambda = std::atof(read_field(it, "regularizationParameter").c_str());
            const int opt = std::atoi(read_field(it, "optimalStepIterationNb").c_str());
            const double thr = huber ? std::atof(read_field(it, "huberThreshold").c_str()) : 0.0;
            const double beta = std::atof(read_field(it, "beta", false, "2").c_str());
            double norms[2] = {0.0, 0.0};
            for (int rep = 0; rep < 2; ++rep)
                die(tomo_regularization_host(0, huber ? TOMO_REG_HUBER : TOMO_REG_GG, vol.data(), out.data(),
                                             c.x_volume_pixel_nb, c.y_volume_pixel_nb, c.z_volume_pixel_nb, lambda,
                                             thr, beta, 1, opt, norms),
                    "getLaplacianRegularizationCriterion");
            std::cout << "jReg = " << norms[0] << std::endl;
        }
        ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        if (!no_save)
            save_raw(op == "laplacien" ? "laplacien.v" : "GG.v", out,
                     {c.z_volume_pixel_nb, c.y_volume_pixel_nb, c.x_volume_pixel_nb});
    } else if (op.empty()) {
        tomo_gradient_params prm{};
        prm.projector = P;
        prm.backprojector = B;
        prm.storage = TOMO_F32;
        prm.gradient_iteration_nb = std::atoi(read_field(it, "gradientIterationNb").c_str());
        prm.optimal_step_iteration_nb = std::atoi(read_field(it, "optimalStepIterationNb").c_str());
        prm.regularization_parameter = std::atof(read_field(it, "regularizationParameter").c_str());
        prm.positivity = std::atoi(read_field(it, "positivity", false, "0").c_str());
        const std::string penalty = read_field(it, "penaltyFunction", false, "GGaussian");
        const std::string grad = read_field(it, "gradient", false, "Simple");
        const double beta = std::atof(read_field(it, "beta", false, "2").c_str());
        // penaltyFunction "Huber" selects the Huber regulariser, anything else the generalised
        // Gaussian with configIteration beta (Iter3D.cu:58-72). gradient "Weighted" runs
        // Iter3D::doWeightedGradient, which the reference's own front end cannot select
        // (Iter3D.cu:77-88 maps Simple, Conjugate and ProjBack): its weight sinogram comes from
        // --weights=<file> (default <workdir>/weightedSinogram.s).
        const bool huber = penalty == "Huber";
        const bool weighted = grad == "Weighted";
        if (grad != "Simple" && !weighted) {
            std::cerr << "available: the simple and the weighted gradient (gradient Simple / Weighted)" << std::endl;
            return EXIT_FAILURE;
        }
        std::vector<float> weights;
        if (weighted) {
            std::string wname = wd + "weightedSinogram.s";
            if (flag(argc, argv, "weights", &v)) wname = v;
            weights.assign(nsino, 0.f);
            if (!load_raw(wname, weights)) {
                std::cerr << "cannot load the weight sinogram " << wname << std::endl;
                return EXIT_FAILURE;
            }
        }
        const double huber_thr = huber ? std::atof(read_field(it, "huberThreshold").c_str()) : 0.0;
        std::vector<float> vol(nvox, 0.f), sino(nsino, 0.f);
        const std::string sname = measured_sinogram();
        if (!load_raw(sname, sino)) {
            std::cerr << "cannot load the sinogram " << sname << std::endl;
            return EXIT_FAILURE;
        }
        const std::string init = read_field(ct, "initVolumeName", false, "none");
        if (init != "none" && !load_raw(init, vol)) {
            std::cerr << "cannot load the initial volume " << init << std::endl;
            return EXIT_FAILURE;
        }
        tomo_solver* sv = nullptr;
        die(tomo_solver_create(ctx, &prm, &sv), "tomo_solver_create");
        if (huber) die(tomo_solver_set_regularizer(sv, TOMO_REG_HUBER, huber_thr), "Huber regulariser");
        else die(tomo_solver_set_gg_beta(sv, beta), "generalised-Gaussian beta");
        if (weighted) die(tomo_solver_set_weights(sv, weights.data(), 1, nullptr), "weight sinogram");
        auto t0 = clk::now();
        die(tomo_solver_iterate_host(sv, vol.data(), sino.data(), 1, prm.gradient_iteration_nb, nullptr),
            weighted ? "doWeightedGradient" : "doSimpleGradient");
        ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        std::vector<double> alpha(prm.gradient_iteration_nb > 0 ? prm.gradient_iteration_nb : 1);
        int32_t n = 0;
        die(tomo_solver_alphas(sv, alpha.data(), (int32_t)alpha.size(), &n, nullptr), "alphas");
        for (int i = 0; i < n; ++i) std::cout << "\titeration " << i + 1 << " alpha = " << alpha[i] << std::endl;
        tomo_solver_destroy(sv);
        if (!no_save) {
            // <workdir>TomoIter/Results/Result_<date>/finalVolume.v (Iter3D.cu:100-118,
            // Iter3D_Algo_Gradient.cu:216)
            char stamp[64];
            const std::time_t now = std::time(nullptr);
            std::strftime(stamp, sizeof(stamp), "TomoIter/Results/Result_%Y_%m_%d_%Hh%M/", std::localtime(&now));
            const std::string outdir = wd + stamp;
            for (const std::string& d : {wd + "TomoIter", wd + "TomoIter/Results", outdir}) ::mkdir(d.c_str(), 0755);
            save_raw(outdir + "finalVolume.v", vol, {c.z_volume_pixel_nb, c.y_volume_pixel_nb, c.x_volume_pixel_nb});
            std::cout << "final volume saved in " << outdir << "finalVolume.v" << std::endl;
        }
    } else {
        std::cerr << "--op=" << op
                  << " is not part of this drop-in (proj, back, back_fdk, laplacien, reg_GG, tiff5, tiff4, or none for"
                     " the gradient)"
                  << std::endl;
        return EXIT_FAILURE;
    }
    std::cout << "Time computation : " << ms << " ms" << std::endl;
    tomo_context_destroy(ctx);
    return 0;
}
