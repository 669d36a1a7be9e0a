// Stand-in for the reference's Image3D_CPU.cuh: a host image of x * y * z values and the
// ImageTiff / ImageCalibration declarations whose definitions the reference's ImageTiff.cu
// supplies (Image3D_CPU.cuh:56-84 interface). Test infrastructure only.
#pragma once
#include <vector>
#include "Config.hpp"

template <typename T> class Image3D_CPU {
public:
    Image3D_CPU(unsigned long x, unsigned long y, unsigned long z) : nx(x), ny(y), data((size_t)x * y * z, T(0)) {}
    T* getImageData() { return data.data(); }
    unsigned long getXImagePixelNb() const { return nx; }
    unsigned long getYImagePixelNb() const { return ny; }
    unsigned long getDataImageSize() const { return (unsigned long)data.size(); }

private:
    unsigned long nx, ny;
    std::vector<T> data;
};

template <typename T> class ImageTiff : public Image3D_CPU<T> {
public:
    ImageTiff(unsigned short xImagePixelNb, unsigned short yImagePixelNb);
    ~ImageTiff();
    void loadTiffImage(string fileName);
};

template <typename T> class ImageCalibration : public ImageTiff<T> {
public:
    ImageCalibration(unsigned short xImagePixelNb, unsigned short yImagePixelNb);
    ~ImageCalibration();
    double getBlackMeanValue();
    double getGrayMeanValue();
    double getWhiteMeanValue(unsigned int CalibrationEnergyNb);
    ImageTiff<T>& getBlackTiffImage();
    ImageTiff<T>& getGrayTiffImage();
    ImageTiff<T>& getWhiteTiffImage();
};
