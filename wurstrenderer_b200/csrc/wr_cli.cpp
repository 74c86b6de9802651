// Command-line front end with the reference's flags (src/main.cpp:5-48):
//   wurst_b200 --simple2parse <scene.json> [--simple2parse <scene2.json> ...]
//   wurst_b200 --jsimple2parse '<scene json text>'
//   wurst_b200            (reads option/"value" pairs from ./default.txt, creating
//                          an empty one when it is missing)
// Unlike the reference, which aborts on an exception, failures print the
// library's error text and return a nonzero exit status.

#include <cstdio>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>

#include "../../include/wurst_b200.h"

static int parse_pair(const std::string &option, const std::string &info) {
    int rc = WR_OK;
    if (option == "--simple2parse") rc = wr_run_simple2(info.c_str());
    else if (option == "--jsimple2parse") rc = wr_run_jsimple2(info.c_str());
    else return WR_OK;   // unknown options are ignored, as in the reference
    if (rc != WR_OK) fprintf(stderr, "wurst_b200: %s (status %d)\n", wr_last_error(), rc);
    return rc;
}

int main(int argc, char **argv) {
    if (argc > 1) {
        for (int i = 1; i + 2 <= argc; i += 2) {
            const int rc = parse_pair(argv[i], argv[i + 1]);
            if (rc != WR_OK) return 1;
        }
        return 0;
    }
    std::ifstream ifs("default.txt");
    if (!ifs.is_open()) {
        std::ofstream ofs("default.txt");
        return 0;
    }
    std::string line;
    while (std::getline(ifs, line)) {
        std::stringstream ss(line);
        std::string option, info;
        ss >> option >> std::quoted(info);
        if (!option.empty() && option[0] != '#' && ss.tellg() != -1) {
            if (parse_pair(option, info) != WR_OK) return 1;
        }
    }
    return 0;
}
