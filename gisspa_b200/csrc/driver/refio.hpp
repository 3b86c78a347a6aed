// Reference-compatible input readers of the drop-in driver.
//
//  - config file   : EMReader/DataReader.cpp:128-265 (key = value, '#' comments)
//  - Euler file    : DataReader.cpp:267-284 ("alt az" per line)
//  - input list    : DataReader.cpp:318-388 (#LST / #LSX), main.cu:125-138 (path prefix)
//  - MRC image     : EMReader/emdata_.cpp:384-617 (modes 0/1/2/4, byte order, sections)
//  - EMAN HDF5     : EMReader/emdata_.cpp:174-199 dispatch, read by gs_hdf_read_image
#pragma once

#include <string>
#include <vector>

namespace gsdrv {

struct Config {
    std::string inlst = "  ", temp2d = "  ", eulerf = "  ";
    float apix = -1, phi_step = -1, kk = -1, energy = -1, cs = -1, highres = -1, lowres = -1, d_m = -1;
    std::string outlst = "./outlst";
    int first = -1, last = -1;
    float thres = 7.0f;
    int device_id = 0, padding_size = 320, phase_flip = 0, overlap = -1, norm_type = 0, invert = 0;
    std::vector<std::string> unknown;  // values of unrecognised keys, as the reference reports them
};

// Parse one "key = value" line the way DataReader.cpp:128-246 splits it.
void parse_config_line(const std::string& line, Config* c);
// Returns false if the file cannot be opened.
bool read_config(const std::string& path, Config* c);
// Names of required keys that are missing (DataReader.cpp:302-315).
std::vector<std::string> missing_required(const Config& c);
void print_config(const Config& c);

struct Euler {
    std::vector<float> alt, az;
};
bool read_euler(const std::string& path, Euler* e);

struct LstEntry {
    int nn = 0;
    std::string path;  // with the list's directory prefixed (as printed in the output)
};
// CTF values persist across entries that do not restate them, like the
// reference's Parameters fields.
struct CtfState {
    float defocus = 0.0f;  // as written in the list (positive underfocus)
    float dfdiff = 0.0f;
    float dfang = 0.0f;
};
// Entry n of the list; returns 1 on success, <0 on the reference's error codes.
int read_lst_entry(const std::string& inlst, int n, LstEntry* out, CtfState* ctf);

struct Image {
    int nx = 0, ny = 0, nz = 0;
    std::vector<float> data;
};
// Section `section` of an MRC file (whole volume if out of range).  Returns
// an empty string on success, otherwise the reason.
std::string read_mrc(const std::string& path, int section, Image* img);
// The file starts with the HDF5 signature (EMhdf::is_valid, emhdf_.cpp:47-62).
bool is_hdf5(const std::string& path);
// emdata::readImage (emdata_.cpp:174-205): image `section` of an EMAN HDF5
// file (gs_hdf_read_image), else section `section` of an MRC file.
std::string read_image(const std::string& path, int section, Image* img);

}  // namespace gsdrv
