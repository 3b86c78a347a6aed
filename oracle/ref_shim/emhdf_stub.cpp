// Link-time stand-ins for the reference's EMhdf / EMhdf2 classes
// (reference EMReader/emhdf_.h, EMReader/emhdf2_.h), whose real bodies need
// the HDF5 1.8 library that is not available here.  is_valid() reports
// "not an HDF file", so emdata::readImage (reference EMReader/emdata_.cpp:174)
// always falls through to readMRC; the remaining members are never reached
// and return failure values.  Test-infrastructure only: this file is part of
// the checker build under oracle/, never of the product.
#include "emhdf_.h"
#include "emhdf2_.h"

EMhdf::EMhdf(const char*, const char*) : file(-1), group(-1), cur_dataset(-1), cur_dataset_id(-1),
                                        old_func(0), old_client_data(0) {}
EMhdf::~EMhdf() {}
int EMhdf::init_test(const char*) { return -1; }
int EMhdf::is_valid(const char*) { return 0; }
int* EMhdf::read_dims(int, int* p_ndim) { if (p_ndim) *p_ndim = 0; return 0; }
int EMhdf::read_data(int, float**) { return -1; }
int EMhdf::read_int_attr(int, const char*) { return 0; }
float EMhdf::read_float_attr(int, const char*) { return 0.0f; }
const char* EMhdf::read_string_attr(int, const char*) { return ""; }
void EMhdf::read_array_attr(int, const char*, void*) {}
int EMhdf::read_euler_attr(int, const char*) { return -1; }
int EMhdf::read_ctfit(int, CTFParam*) { return -1; }
int EMhdf::read_mapinfo_attr(int, const char*) { return -1; }

EMhdf2::EMhdf2(const char*, const char*) : file(-1), group(-1), accprop(-1), simple_space(-1),
                                          initialized(false), rwmode("r") {}
EMhdf2::~EMhdf2() {}
emdataHeader* EMhdf2::read_header(int, Euler&) { return 0; }
int EMhdf2::read_data(float*, int) { return -1; }
