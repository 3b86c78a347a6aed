// gisspa_merge: drop-in for the reference's
// python_scripts/remove_repeat_particles_from_list.py
//     gisspa_merge <input.lst> <number of images> <center thres> <euler thres> <output.lst>
// Reads the pick lines, groups runs of one micrograph path (field 2), merges
// duplicates with gs_merge_duplicates on GPU 0 and writes the kept lines
// unchanged and in order.  <number of images> is accepted for the script's
// argument order; the script uses it only to size its tables.
#include "gisspa.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <string>
#include <vector>

static std::vector<std::string> split(const std::string& s, char c) {
    std::vector<std::string> out;
    size_t a = 0;
    for (;;) {
        const size_t b = s.find(c, a);
        out.push_back(s.substr(a, b == std::string::npos ? std::string::npos : b - a));
        if (b == std::string::npos) break;
        a = b + 1;
    }
    return out;
}

// "key=v0,v1,..." -> values
static std::vector<double> values(const std::string& field) {
    std::vector<double> v;
    const size_t eq = field.find('=');
    if (eq == std::string::npos) return v;
    for (const std::string& t : split(field.substr(eq + 1), ',')) v.push_back(strtod(t.c_str(), nullptr));
    return v;
}

int main(int argc, char** argv) {
    if (argc < 6) {
        printf("<input1> <number of images> <center> <euler_thres> <output>\n");
        return 1;
    }
    const double center = strtod(argv[3], nullptr), thres = strtod(argv[4], nullptr);
    std::ifstream in(argv[1], std::ios::binary);
    if (!in) {
        fprintf(stderr, "cannot read %s\n", argv[1]);
        return 2;
    }
    // lines with their own line ends (a last line without one stays so)
    const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    std::vector<std::string> lines;
    for (size_t a = 0; a < text.size();) {
        const size_t b = text.find('\n', a);
        const size_t e = b == std::string::npos ? text.size() : b + 1;
        lines.push_back(text.substr(a, e - a));
        a = e;
    }
    std::vector<gs_merge_item> items(lines.size());
    long long group = -1;
    std::string prev;
    for (size_t k = 0; k < lines.size(); ++k) {
        std::string body = lines[k];
        if (!body.empty() && body.back() == '\n') body.pop_back();
        const std::vector<std::string> f = split(body, '\t');
        if (f.size() < 8) {
            fprintf(stderr, "line %zu: expected 8 tab-separated fields\n", k + 1);
            return 2;
        }
        if (k == 0 || f[1] != prev) ++group;
        prev = f[1];
        const std::vector<double> e = values(f[5]), c = values(f[6]), s = values(f[7]);
        if (e.size() < 3 || c.size() < 2 || s.empty()) {
            fprintf(stderr, "line %zu: malformed euler/center/score field\n", k + 1);
            return 2;
        }
        items[k] = gs_merge_item{c[0], c[1], e[0], e[1], e[2], s[0], group};
    }
    std::vector<unsigned char> keep(lines.size(), 1);
    const int st = gs_merge_duplicates(0, items.data(), items.size(), center, thres, keep.data());
    if (st != GS_OK) {
        fprintf(stderr, "gs_merge_duplicates: %s\n", gs_status_string(st));
        return 3;
    }
    FILE* out = fopen(argv[5], "w");
    if (!out) {
        fprintf(stderr, "cannot write %s\n", argv[5]);
        return 2;
    }
    for (size_t k = 0; k < lines.size(); ++k)
        if (keep[k]) fputs(lines[k].c_str(), out);
    fclose(out);
    return 0;
}
