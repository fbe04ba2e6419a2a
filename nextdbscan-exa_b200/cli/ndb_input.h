// ndb_input.h -- input readers of nextdbscan-exa (magma_input.h) for one rank, host side.
//
//   .bin  int32 n, int32 d, float32[n*d] row-major (magma_input.h:113-125)
//   .csv  one point per line, space separated, atof then cast to float; the
//         dimension count is the token count of the first line (magma_input.h:53-67,
//         :127-142, :161-165)
//   .h5 / .hdf5  not supported by this build: error and exit(-1), as the reference
//         does without HDF5_ON (magma_input.h:152-160)
// Unlike the reference reader, a short or unreadable file is reported instead of
// being read as zeros.
#ifndef NDB_INPUT_H
#define NDB_INPUT_H

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace ndb_input {

inline bool ends_with(const std::string &s, const std::string &suffix) {
    return s.size() >= suffix.size() && s.compare(s.size() - suffix.size(), suffix.size(), suffix) == 0;
}

inline bool read_bin(const std::string &path, std::vector<float> &v, int &n, int &d) {
    std::ifstream ifs(path, std::ios::in | std::ios::binary);
    if (!ifs) {
        std::cerr << "Error: cannot open " << path << std::endl;
        return false;
    }
    int32_t hdr[2] = {0, 0};
    ifs.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    if (ifs.gcount() != (std::streamsize)sizeof(hdr) || hdr[0] < 0 || hdr[1] <= 0) {
        std::cerr << "Error: bad .bin header in " << path << std::endl;
        return false;
    }
    n = hdr[0];
    d = hdr[1];
    v.resize((size_t)n * (size_t)d);
    ifs.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(v.size() * sizeof(float)));
    if (ifs.gcount() != (std::streamsize)(v.size() * sizeof(float))) {
        std::cerr << "Error: " << path << " holds fewer than n*d floats" << std::endl;
        return false;
    }
    return true;
}

inline bool read_csv(const std::string &path, std::vector<float> &v, int &n, int &d) {
    std::ifstream is(path);
    if (!is) {
        std::cerr << "Error: cannot open " << path << std::endl;
        return false;
    }
    std::string line, tok;
    n = 0;
    d = 0;
    v.clear();
    while (std::getline(is, line)) {
        std::istringstream ss(line);
        if (d == 0) {
            while (ss >> tok) ++d;
            ss.clear();
            ss.str(line);
        }
        for (int j = 0; j < d; ++j) {
            ss >> tok;
            v.push_back(static_cast<float>(std::atof(tok.c_str())));
        }
        ++n;
    }
    std::cout << "WARNING: USING SLOW CSV I/O." << std::endl;
    return d > 0;
}

inline bool read_input(const std::string &path, std::vector<float> &v, int &n, int &d) {
    if (ends_with(path, ".bin")) return read_bin(path, v, n, d);
    if (ends_with(path, ".h5") || ends_with(path, ".hdf5")) {
        std::cerr << "Error: HDF5 is not supported by this executable." << std::endl;
        std::exit(-1);
    }
    if (ends_with(path, ".csv")) return read_csv(path, v, n, d);
    std::cerr << "Error: unsupported input type " << path << std::endl;
    return false;
}

}  // namespace ndb_input

#endif  // NDB_INPUT_H
