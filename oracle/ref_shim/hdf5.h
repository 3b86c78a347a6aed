/* Minimal stand-in for the HDF5 1.8 C header, used ONLY to compile the
 * reference GisSPA sources (EMReader/emhdf_.h, emhdf2_.h) into the parity
 * checker under oracle/_ref.  It declares the three handle types those
 * headers name; no HDF5 function is declared or called.  Every HDF input
 * path of the reference is routed away by the stub EMhdf::is_valid()
 * (oracle/ref_shim/emhdf_stub.cpp), so all inputs go through readMRC. */
#ifndef GISSPA_REF_SHIM_HDF5_H
#define GISSPA_REF_SHIM_HDF5_H
typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
#endif
