// SPDX-License-Identifier: 0BSD
// Test driver: the reference's --manifest command line (--manifest=FILE,
// --tend=SECONDS) over include/manifest.hpp, printing the reference's header
// comment and RESULT lines; exit status 4 for an unusable manifest, 1 for a
// CUDA failure.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "manifest.hpp"

int main(int argc, char** argv) {
    std::string path;
    double t_end = 1.5e-3;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a.rfind("--manifest=", 0) == 0) path = a.substr(11);
        else if (a.rfind("--tend=", 0) == 0) t_end = std::atof(a.c_str() + 7);
    }
    std::vector<lpbf::manifest::RunSpec> rows;
    std::string err;
    if (!lpbf::manifest::read_manifest(path, &rows, &err)) {
        std::fprintf(stderr, "%s\n", err.c_str());
        return 4;
    }
    lpbf::manifest::print_header(stdout);
    std::vector<lpbf::manifest::RowResult> res;
    const bool ok = lpbf::manifest::run_rows(rows, t_end, &res);
    for (size_t i = 0; i < rows.size(); ++i) lpbf::manifest::print_result(stdout, rows[i], res[i]);
    std::fprintf(stderr, "[manifest] completed %zu runs\n", rows.size());
    return ok ? 0 : 1;
}
