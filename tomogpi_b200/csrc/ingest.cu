// ingest.cu -- real-data ingest (host only): the normalised negative-log sinogram that the
// reference builds from its detector files (ConfigTiff<unsigned short>::
// createNormalizedMeanNegativeLogSinogram_5dig / _4dig, inc/Config/ConfigTiff.hpp:287-420,
// --op=tiff5 / tiff4, Iter3D_main.cu:317-336).
//
// File format, as the reference reads it: a header of four 16-bit words, then the image
// row-major in 16-bit unsigned words (ImageTiff::loadTiffImage, ImageTiff.cu:18-38). The
// white level is the mean of the last 1/E of the calibration image's rows (E energies,
// ImageCalibration::getWhiteMeanValue, ImageTiff.cu:81-94). Projections are read from file
// number total + 1 down in steps of rate = total / used (used files), each cropped to the
// final detector window around its centre, every pixel mapped to -log(value / white) in FP32.
// A few MB per view of byte reading and one log per pixel: host work by nature (the files
// arrive through the host), so no device code here.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "tomo_common.cuh"

using namespace tomo;

namespace {

bool read_image(const std::string& path, size_t count, std::vector<unsigned short>& out) {
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f.is_open()) return false;
    unsigned short header[4];
    f.read(reinterpret_cast<char*>(header), sizeof(header));
    out.resize(count);
    f.read(reinterpret_cast<char*>(out.data()), (std::streamsize)(count * sizeof(unsigned short)));
    return (size_t)f.gcount() == count * sizeof(unsigned short);
}

}  // namespace

extern "C" {

tomo_status tomo_tiff_white_mean(const char* calibration_file, int32_t nx, int32_t ny, int32_t energy_nb, double* mean) {
    TOMO_CHECK_ARG(calibration_file && mean && nx > 0 && ny > 0 && energy_nb > 0, "tomo_tiff_white_mean: bad argument");
    std::vector<unsigned short> img;
    if (!read_image(calibration_file, (size_t)nx * ny, img)) {
        set_error(std::string("tomo_tiff_white_mean: cannot read ") + calibration_file);
        return TOMO_ERR_IO;
    }
    double s = 0.0;
    for (int y = (energy_nb - 1) * ny / energy_nb; y < ny; ++y)  // integer row bound (ImageTiff.cu:87)
        for (int x = 0; x < nx; ++x) s += img[(size_t)x + (size_t)y * nx];
    *mean = s / ((double)nx * ny / (double)energy_nb);         // :91
    return TOMO_OK;
}

tomo_status tomo_tiff_negative_log_sinogram(const tomo_tiff_config* c, const char* tif_dir, const char* tiff_name,
                                            const char* calibration_file, float* sinogram) {
    TOMO_CHECK_ARG(c && tif_dir && tiff_name && calibration_file && sinogram, "tomo_tiff_negative_log_sinogram: null argument");
    TOMO_CHECK_ARG(c->used_projection_nb > 0 && c->total_projection_nb >= c->used_projection_nb &&
                       c->u_initial_nb > 0 && c->v_initial_nb > 0 && c->u_final_nb > 0 && c->v_final_nb > 0 &&
                       (c->digits == 4 || c->digits == 5),
                   "tomo_tiff_negative_log_sinogram: bad configuration");
    double white = 0.0;
    tomo_status s = tomo_tiff_white_mean(calibration_file, c->u_calibration_nb, c->v_calibration_nb,
                                         c->calibration_energy_nb, &white);
    if (s != TOMO_OK) return s;
    const float wf = (float)white;  // calibrationImageMeanValue is a float (ConfigTiff.hpp:305)
    // unsigned short window bounds (ConfigTiff.hpp:294-297)
    const unsigned short inf_u = (unsigned short)(c->u_center_final - c->u_final_nb / 2);
    const unsigned short inf_v = (unsigned short)(c->v_center_final - c->v_final_nb / 2);
    const unsigned short sup_u = (unsigned short)(c->u_center_final + c->u_final_nb / 2);
    const unsigned short sup_v = (unsigned short)(c->v_center_final + c->v_final_nb / 2);
    const int rate = c->total_projection_nb / c->used_projection_nb;  // ConfigTiff.cpp:24
    const size_t nu = c->u_final_nb, nv = c->v_final_nb;
    // window pixels outside the file keep 0 (the reference leaves them unwritten)
    std::fill(sinogram, sinogram + nu * nv * (size_t)c->used_projection_nb, 0.f);
    std::vector<unsigned short> img;
    int phi = 0;
    for (int p = c->total_projection_nb; p > c->total_projection_nb - rate * c->used_projection_nb; p -= rate) {
        char num[32];
        std::snprintf(num, sizeof(num), c->digits == 5 ? "_%05d.tif" : "_%04d.tif", p + 1);
        const std::string path = std::string(tif_dir) + "/" + tiff_name + num;
        if (!read_image(path, (size_t)c->u_initial_nb * c->v_initial_nb, img)) {
            set_error("tomo_tiff_negative_log_sinogram: cannot read " + path);
            return TOMO_ERR_IO;
        }
        for (int v = 0; v < c->v_initial_nb; ++v)
            for (int u = 0; u < c->u_initial_nb; ++u) {
                if (!(v >= inf_v && u >= inf_u && v < sup_v && u < sup_u)) continue;
                const float ratio = (float)img[(size_t)v * c->u_initial_nb + u] / wf;
                sinogram[(size_t)(u - inf_u) + (size_t)(v - inf_v) * nu + (size_t)phi * nu * nv] = -std::log(ratio);
            }
        ++phi;
    }
    return TOMO_OK;
}

}  // extern "C"
