// merge_renderings -- helperScripts/mergeMultipleRenderings.cpp's command line over the library's
// host layer, with the mean weighted by photon counts:
//
//   merge_renderings prefix=P renderings=R pathLengthBins=B [photons=N0,N1,...]
//       reads P_<i>_<j>.pfm (i < R, j < B), writes P_mean_<j>.pfm
//   merge_renderings pfm3d out.pfm3d in0.pfm3d[:N0] in1.pfm3d[:N1] ...
//       merges PFM3D films (renderer3d / simplER outputs)
//
// Without photon counts every rendering weighs the same (the plain mean; the reference helper's
// running mean gives its first rendering extra weight).
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>

#include "smp_host.h"

static std::vector<std::string> split(const std::string &s, char d) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string t;
    while (std::getline(ss, t, d)) if (!t.empty()) out.push_back(t);
    return out;
}

int main(int argc, char **argv) {
    std::string err;
    if (argc > 1 && std::strcmp(argv[1], "pfm3d") == 0) {
        if (argc < 4) { std::cerr << "usage: merge_renderings pfm3d out.pfm3d in.pfm3d[:photons] ...\n"; return -1; }
        std::vector<std::vector<double>> films;
        std::vector<double> w;
        int X = 0, Y = 0, Z = 0;
        for (int i = 3; i < argc; ++i) {
            std::string a = argv[i];
            double n = 1.0;
            size_t c = a.rfind(':');
            if (c != std::string::npos && c + 1 < a.size() && a.find(".pfm3d", c) == std::string::npos) {
                n = std::atof(a.c_str() + c + 1);
                a = a.substr(0, c);
            }
            int x, y, z;
            films.emplace_back();
            if (!smp_host::read_pfm3d(a, x, y, z, films.back(), err)) { std::cerr << err << std::endl; return -1; }
            if (i > 3 && (x != X || y != Y || z != Z)) { std::cerr << "film sizes differ: " << a << std::endl; return -1; }
            X = x; Y = y; Z = z;
            w.push_back(n);
        }
        std::vector<const std::vector<double> *> ptrs;
        for (auto &f : films) ptrs.push_back(&f);
        std::vector<double> out;
        if (!smp_host::merge_films(ptrs, w, out, err) || !smp_host::write_pfm3d(argv[2], X, Y, Z, out.data(), err)) {
            std::cerr << err << std::endl;
            return -1;
        }
        return 0;
    }
    std::string prefix = "../renderings/complexTiming";
    int renderings = 2, bins = 4096;
    std::vector<double> photons;
    for (int i = 1; i < argc; ++i) {
        std::vector<std::string> p = split(argv[i], '=');
        if (p.size() != 2) { std::cerr << "Input argument " << argv[i] << " should be in the format arg=value" << std::endl; return -1; }
        if (p[0] == "prefix") prefix = p[1];
        else if (p[0] == "renderings") renderings = std::atoi(p[1].c_str());
        else if (p[0] == "pathLengthBins") bins = std::atoi(p[1].c_str());
        else if (p[0] == "photons") for (auto &t : split(p[1], ',')) photons.push_back(std::atof(t.c_str()));
        else {
            std::cerr << "Unknown variable in the input argument:" << p[0] << std::endl
                      << "Should be one of prefix renderings pathLengthBins photons" << std::endl;
            return -1;
        }
    }
    if (!smp_host::merge_reference_bins(prefix, renderings, bins, photons, err)) { std::cerr << err << std::endl; return -1; }
    return 0;
}
