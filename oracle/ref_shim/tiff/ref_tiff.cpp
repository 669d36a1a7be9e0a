// C entry points over the reference's own detector-file ingest, compiled on the host for the
// oracle (ConfigTiff<unsigned short>::createNormalizedMeanNegativeLogSinogram_5dig / _4dig,
// ConfigTiff.hpp:287-420; ImageCalibration::getWhiteMeanValue, ImageTiff.cu:81-94).
// `config_dir` ends with '/' (the reference concatenates it with "configTiff"). Test
// infrastructure only.
#include <cstring>
#include "ConfigTiff.hpp"

extern "C" {

long ref_tiff_sinogram(const char* config_dir, int digits, float* out, long capacity) {
    ConfigTiff<unsigned short> cfg(config_dir, "configTiff");
    Sinogram3D_CPU<float>& s = digits == 4 ? cfg.createNormalizedMeanNegativeLogSinogram_4dig<float>()
                                           : cfg.createNormalizedMeanNegativeLogSinogram_5dig<float>();
    const long n = (long)s.size();
    if (n <= capacity) std::memcpy(out, s.getDataSinogram(), sizeof(float) * n);
    delete &s;
    return n;
}

double ref_tiff_white_mean(const char* file, int nx, int ny, int energy_nb) {
    ImageCalibration<unsigned short> img((unsigned short)nx, (unsigned short)ny);
    img.loadTiffImage(file);
    return img.getWhiteMeanValue((unsigned)energy_nb);
}
}
