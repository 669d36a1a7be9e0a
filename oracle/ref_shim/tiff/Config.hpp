// Stand-in for the reference's Config.hpp when its detector-file ingest (ConfigTiff.hpp,
// ConfigTiff.cpp, ImageTiff.cu) is compiled on the host for the oracle: the configuration
// file reader only (Config.hpp:38-56 interface), without the volume, detector and CUDA
// class tree the full header pulls in. Test infrastructure only.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
using namespace std;

class CUDAArchitecture;

class Config {
public:
    Config() {}
    Config(string dir, string file) : configFileName(file), configDirectoryName(dir) {}
    string getConfigDirectoryName() const { return configDirectoryName; }
    // first whitespace-separated token equal to `field`, then the next token (Config.cpp:35-69)
    template <typename T> T getConfigFileField(string field) {
        ifstream f((configDirectoryName + configFileName).c_str());
        string row, tok;
        while (f && getline(f, row)) {
            istringstream ss(row);
            while (ss >> tok) {
                if (tok == field) {
                    T v{};
                    ss >> v;
                    return v;
                }
            }
        }
        cout << "Unable to find field " << field << endl;
        exit(EXIT_FAILURE);
    }

private:
    string configFileName;
    string configDirectoryName;
};
