#include "refio.hpp"

#include "gisspa.h"

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <utility>

namespace gsdrv {

void parse_config_line(const std::string& line, Config* c) {
    size_t i = 0;
    while (i < line.size() && line[i] != ' ' && line[i] != '=') ++i;
    const std::string option = line.substr(0, i);
    while (i < line.size() && (line[i] == ' ' || line[i] == '=')) ++i;
    const std::string value = line.substr(i);
    const char* v = value.c_str();
    if (option == "input") c->inlst = value;
    else if (option == "template") c->temp2d = value;
    else if (option == "eulerfile") c->eulerf = value;
    else if (option == "kk") c->kk = (float)atof(v);
    else if (option == "angpix") c->apix = (float)atof(v);
    else if (option == "phistep") c->phi_step = (float)atof(v);
    else if (option == "energy") c->energy = (float)atof(v);
    else if (option == "cs") c->cs = (float)atof(v);
    else if (option == "Highres") c->highres = (float)atof(v);
    else if (option == "Lowres") c->lowres = (float)atof(v);
    else if (option == "diameter") c->d_m = (float)atof(v);
    else if (option == "output") c->outlst = value;
    else if (option == "first") c->first = atoi(v);
    else if (option == "last") c->last = atoi(v);
    else if (option == "threshold") c->thres = (float)atof(v);
    else if (option == "GPU_ID") c->device_id = atoi(v);
    else if (option == "window_size") c->padding_size = atoi(v);
    else if (option == "phase_flip") c->phase_flip = atoi(v);
    else if (option == "overlap") c->overlap = atoi(v);
    else if (option == "norm_type") c->norm_type = atoi(v);
    else if (option == "invert") c->invert = atoi(v);
    else c->unknown.push_back(value);
}

bool read_config(const std::string& path, Config* c) {
    std::ifstream f(path);
    if (!f) return false;
    std::string buf;
    while (std::getline(f, buf)) {
        if (buf.empty() || buf[0] == '#') continue;
        parse_config_line(buf, c);
    }
    return true;
}

std::vector<std::string> missing_required(const Config& c) {
    std::vector<std::string> m;
    if (c.inlst[0] == ' ') m.push_back("input");
    if (c.temp2d[0] == ' ') m.push_back("template");
    if (c.eulerf[0] == ' ') m.push_back("eulerfile");
    if (c.apix < 0) m.push_back("angpix");
    if (c.phi_step < 0) m.push_back("phistep");
    if (c.kk < 0) m.push_back("kk");
    if (c.energy < 0) m.push_back("energy");
    if (c.cs < 0) m.push_back("cs");
    if (c.highres < 0) m.push_back("Highres");
    if (c.lowres < 0) m.push_back("Lowres");
    if (c.d_m < 0) m.push_back("diameter");
    return m;
}

void print_config(const Config& c) {
    printf("Parameter requested:\n");
    printf("--input            %s\n", c.inlst.c_str());
    printf("--template         %s\n", c.temp2d.c_str());
    printf("--eulerfile        %s\n", c.eulerf.c_str());
    printf("--angpix           %f\n", c.apix);
    printf("--phistep          %f\n", c.phi_step);
    printf("--kk               %f\n", c.kk);
    printf("--energy           %f\n", c.energy);
    printf("--cs               %f\n", c.cs);
    printf("--Highres          %f\n", c.highres);
    printf("--Lowres           %f\n", c.lowres);
    printf("--diameter         %f\n", c.d_m);
    printf("Parameter optional:\n");
    printf("--threshold        %f\n", c.thres);
    printf("--output           %s\n", c.outlst.c_str());
    printf("--first            %d\n", c.first);
    printf("--last             %d\n", c.last);
    printf("--window_size      %d\n", c.padding_size);
    printf("--GPU_ID           %d\n", c.device_id);
    printf("--phase_flip       %d\n", c.phase_flip);
    printf("--overlap          %d\n", c.overlap);
    printf("--norm_type        %d\n", c.norm_type);
    printf("--invert           %d\n\n", c.invert);
}

bool read_euler(const std::string& path, Euler* e) {
    std::ifstream f(path);
    if (!f) return false;
    std::string buf;
    while (std::getline(f, buf)) {
        if (buf.empty() || buf[0] == '#') continue;
        float a = 0.0f, z = 0.0f;
        sscanf(buf.c_str(), "%f %f", &a, &z);
        e->alt.push_back(a);
        e->az.push_back(z);
    }
    return true;
}

static void parse_pairs(const char* rest, CtfState* ctf) {
    // whitespace-separated key=value tokens (util_func.cpp:27-76 Split,
    // DataReader.cpp:366-388)
    const char* p = rest;
    while (*p) {
        while (*p && isspace((unsigned char)*p)) ++p;
        const char* s = p;
        while (*p && !isspace((unsigned char)*p)) ++p;
        std::string tok(s, p - s);
        float v;
        if (tok.compare(0, 8, "defocus=") == 0) {
            if (sscanf(tok.c_str() + 8, "%f", &v) == 1) ctf->defocus = v;
        } else if (tok.compare(0, 7, "dfdiff=") == 0) {
            if (sscanf(tok.c_str() + 7, "%f", &v) == 1) ctf->dfdiff = v;
        } else if (tok.compare(0, 6, "dfang=") == 0) {
            if (sscanf(tok.c_str() + 6, "%f", &v) == 1) ctf->dfang = v;
        }
    }
}

int read_lst_entry(const std::string& inlst, int n, LstEntry* out, CtfState* ctf) {
    const int kMax = 1024 + 10;
    std::vector<char> buf(kMax);
    std::vector<char> name(kMax), rest(kMax);
    FILE* in = fopen(inlst.c_str(), "rb");
    if (!in) return -3;
    if (!fgets(buf.data(), kMax, in)) { fclose(in); return 0; }
    int nn = 0;
    name[0] = 0;
    rest[0] = 0;
    if (strncmp(buf.data(), "#LSX", 4) == 0) {
        int step = 0;
        if (!fgets(buf.data(), kMax, in) || !fgets(buf.data(), kMax, in)) { fclose(in); return 0; }
        sscanf(buf.data() + 1, " %d", &step);
        if (step == 0) { fclose(in); return -1; }
        const long tl = ftell(in);
        if (n > 0) fseek(in, (long)step * n, SEEK_CUR);
        if (!fgets(buf.data(), kMax, in)) { fclose(in); return -2; }
        if ((ftell(in) - tl) % step != 0) { fclose(in); return -3; }
        sscanf(buf.data(), " %d %1033s %1033[^\n]", &nn, name.data(), rest.data());
        fclose(in);
    } else {
        if (n < 0) n = 0;
        int i;
        for (i = 0; i <= n; ++i) {
            if (!fgets(buf.data(), kMax, in)) break;
            if (buf[0] == '#') --i;
            else {
                rest[0] = 0;
                sscanf(buf.data(), " %d %1033s %1033[^\n]", &nn, name.data(), rest.data());
            }
        }
        fclose(in);
        if (i <= n) return -1;
    }
    parse_pairs(rest.data(), ctf);
    const size_t slash = inlst.rfind('/');
    out->nn = nn;
    out->path = (slash == std::string::npos ? std::string() : inlst.substr(0, slash + 1)) + name.data();
    return 1;
}

static void bswap4(void* p) {
    unsigned char* c = (unsigned char*)p;
    std::swap(c[0], c[3]);
    std::swap(c[1], c[2]);
}

std::string read_mrc(const std::string& path, int section, Image* img) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return "cannot open MRC file " + path;
    unsigned char hdr[1024];
    if (fread(hdr, 1, 1024, f) != 1024) { fclose(f); return "short MRC header in " + path; }
    const bool swap = hdr[0] == 0 && hdr[1] == 0;  // file is big-endian (emdata_.cpp:451-458)
    int32_t w[56];
    memcpy(w, hdr, sizeof w);
    if (swap) for (int k = 0; k < 56; ++k) bswap4(&w[k]);
    int nx = w[0], ny = w[1], nz = w[2];
    const int mode = w[3];
    const int nsymbt = w[23];
    const int nlabl = w[55];
    if (ny > 0xffff || nz > 0xffff || mode > 4 || nlabl > 11 || nx <= 0 || ny <= 0 || nz <= 0) {
        fclose(f);
        return "invalid MRC file " + path;
    }
    if (ny == 1) { fclose(f); return "1D MRC file " + path; }
    if (mode == 3) { fclose(f); return "short-complex MRC input is not supported: " + path; }
    if (mode == 4) nx *= 2;
    int z0 = 0, zn = nz;
    if (section >= 0 && section < nz) { z0 = section; zn = 1; }
    const size_t esz = mode == 0 ? 1 : (mode == 1 ? 2 : 4);
    const size_t count = (size_t)nx * ny * zn;
    std::vector<unsigned char> raw(count * esz);
    if (fseek(f, 1024 + nsymbt + (long)((size_t)z0 * nx * ny * esz), SEEK_SET) != 0 ||
        fread(raw.data(), esz, count, f) != count) {
        fclose(f);
        return "truncated MRC data in " + path;
    }
    fclose(f);
    img->nx = nx;
    img->ny = ny;
    img->nz = zn;
    img->data.resize(count);
    for (size_t i = 0; i < count; ++i) {
        const unsigned char* p = raw.data() + i * esz;
        if (mode == 0) {
            img->data[i] = (float)((double)p[0] / 100.0 - 1.28);
        } else if (mode == 1) {
            int16_t s;
            memcpy(&s, p, 2);
            if (swap) s = (int16_t)(((uint16_t)s >> 8) | ((uint16_t)s << 8));
            img->data[i] = (float)s;
        } else {
            float v;
            memcpy(&v, p, 4);
            if (swap) bswap4(&v);
            img->data[i] = v;
        }
    }
    return "";
}

bool is_hdf5(const std::string& path) {
    static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    unsigned char s[8] = {0};
    const bool ok = fread(s, 1, 8, f) == 8 && memcmp(s, sig, 8) == 0;
    fclose(f);
    return ok;
}

std::string read_image(const std::string& path, int section, Image* img) {
    if (!is_hdf5(path)) return read_mrc(path, section, img);
    float* data = nullptr;
    int nx = 0, ny = 0, nz = 0;
    char err[512];
    const int st = gs_hdf_read_image(path.c_str(), section, &data, &nx, &ny, &nz, err, sizeof err);
    if (st != GS_OK) return std::string(err[0] ? err : gs_status_string(st));
    img->nx = nx;
    img->ny = ny;
    img->nz = nz;
    img->data.assign(data, data + (size_t)nx * ny * nz);
    gs_host_free(data);
    return "";
}

}  // namespace gsdrv
