// renderer3d -- the key=value front-end of renderer/samples/renderer3d_sample.cpp over the B200
// march. Same keys, defaults, strict mode and sanity checks; writes <outFilePrefix>.pfm3d.
// "--dry-run" as the first argument parses and prints the resolved inputs and descriptors
// without rendering (no GPU needed).
#include <cstring>
#include <iostream>

#include "smp_host.h"

int main(int argc, char **argv) {
    bool dry = argc > 1 && std::strcmp(argv[1], "--dry-run") == 0;
    if (dry) { argv[1] = argv[0]; ++argv; --argc; }
    smp_host::RenderConfig cfg;
    std::string err;
    if (smp_host::parse_cli(argc, argv, cfg, err) != 0) {
        std::cerr << err << std::endl;
        return -1;
    }
    if (cfg.printInputs) smp_host::print_inputs(cfg, std::cout);
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
