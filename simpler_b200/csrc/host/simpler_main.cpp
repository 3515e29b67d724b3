// simplER -- the JSON-settings front-end of simplER.cpp over the B200 march: reads the settings
// file (argv[1], default config.json; the layout of renderer/src/settings_parser.cpp) and writes
// <rendering_type>_<YYYY_MM_DD_HH_MM>.pfm3d. "--dry-run" before the file name parses and prints
// the resolved descriptors without rendering (no GPU needed).
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>

#include "smp_host.h"

int main(int argc, char **argv) {
    int a = 1;
    bool dry = argc > a && std::strcmp(argv[a], "--dry-run") == 0;
    if (dry) ++a;
    std::string path = argc > a ? argv[a] : "config.json";
    std::cout << "Using config file: " << path << std::endl;
    std::ifstream f(path);
    if (!f.is_open()) {
        std::cerr << "Failed to open " << path << std::endl;
        return 1;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    smp_host::Json root;
    std::string err;
    if (!smp_host::parse_json(ss.str(), root, err) || root.kind != smp_host::Json::Object) {
        std::cerr << "Failed to parse " << path << ": " << (err.empty() ? "top-level JSON must be an object" : err) << std::endl;
        return 1;
    }
    smp_host::RenderConfig cfg;
    if (smp_host::parse_json_settings(root, cfg, err) != 0) {
        std::cerr << err << std::endl;
        return 1;
    }
    if (cfg.printInputs) {
        std::cout << "simplER renderer started with the following parameters:\n";
        smp_host::print_inputs(cfg, std::cout);
    }
    if (dry) {
        smp_host::Built b;
        int rc = smp_host::build_descs(cfg, b, err);
        if (rc) { std::cerr << err << std::endl; return 1; }
        smp_host::print_descs(b, std::cout);
        std::cout << "output = " << cfg.outputFile << std::endl;
        return 0;
    }
    int rc = smp_host::run(cfg, std::cout, err);
    if (rc) { std::cerr << "render failed (" << rc << "): " << err << std::endl; return 1; }
    return 0;
}
