// Uses the C++ drop-in header as the reference's callers use its operator classes
// (Iter3D_main.cu:78,108, Iter3D_Algo_Gradient.cu:80,106): the argument is an output
// directory; the program reads volume.v (32^3) and writes the operators' outputs there.
#include <cstdio>
#include <string>

#include "tomogpi_b200/TomoGPI.hpp"

using namespace tomogpi;

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    const unsigned long n = 32, P = 24;
    UniformAcquisition acq(128.0, 64.0, 0.0, 2.0, 0.0, P);   // FDD, FOD, start, stop (units of pi)
    Detector det(64.f, 64.f, n, n);                          // pitch 2
    try {
        Volume_CPU<float> vol(32.f, 32.f, 32.f, n, n, n);
        vol.loadVolume(dir + "/volume.v");
        Sinogram3D_CPU<float> sino(n, n, P);
        CUDAProjectionArchitecture pa;
        CUDABProjectionArchitecture ba;
        RegularSamplingProjector_compute_CUDA_mem_CPU<float> rs(&acq, &det, &pa, &vol);
        rs.doProjection(&sino, &vol);
        sino.saveSinogram(dir + "/rs.s");
        SiddonProjector_compute_C_mem_CPU<float> sid(&acq, &det, &vol);
        Sinogram3D_CPU<float> sino2(n, n, P);
        sid.doProjection(&sino2, &vol);
        sino2.saveSinogram(dir + "/siddon.s");
        Volume_CPU<float> back(32.f, 32.f, 32.f, n, n, n);
        VIBackProjector_compute_CUDA_mem_CPU<float> vi(&acq, &det, &ba, &back, 0);
        vi.doBackProjection(&back, &sino);
        back.saveVolume(dir + "/vi.v");
        vi.setFdk(1);
        vi.doBackProjection(&back, &sino);
        back.saveVolume(dir + "/fdk.v");
        // mem_GPU: managed buffers
        Volume_GPU<float> gvol(32.f, 32.f, 32.f, n, n, n);
        std::copy(vol.getVolumeData(), vol.getVolumeData() + n * n * n, gvol.getVolumeData());
        Sinogram3D_GPU<float> gsino(n, n, P);
        RegularSamplingProjector_compute_CUDA_mem_GPU<float> rsu(&acq, &det, &pa, &gvol);
        rsu.doProjection(&gsino, &gvol);
        Volume_CPU<float>::save_raw(dir + "/rs_um.s", gsino.getDataSinogram(), n * n * P);
        Volume_GPU<float> gback(32.f, 32.f, 32.f, n, n, n);
        VIBackProjector_compute_CUDA_mem_GPU<float> viu(&acq, &det, &ba, &gback, 0);
        viu.doBackProjection(&gback, &gsino);
        Volume_CPU<float>::save_raw(dir + "/vi_um.v", gback.getVolumeData(), n * n * n);
        // errors surface as exceptions, not exit()
        try {
            Volume_CPU<float> missing(32.f, 32.f, 32.f, n, n, n);
            missing.loadVolume(dir + "/no_such_file.v");
            return 3;
        } catch (const Error&) {
        }
    } catch (const Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
