/*
 * Type, constant and prototype stubs so that the reference headers that include
 * <hdf5.h> (util.h) and its test programs compile without libhdf5.  The oracle
 * builds use the types only; the reference's C test programs get H5Fopen /
 * H5Fclose and the util.h read helpers from h5_npz.c, which serves the .npz
 * fixtures.  TEST INFRASTRUCTURE ONLY.
 */
#pragma once
#include <stdint.h>
typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

#define H5F_ACC_RDONLY 0u
#define H5F_ACC_TRUNC 2u
#define H5P_DEFAULT ((hid_t)0)
#define H5T_NATIVE_DOUBLE ((hid_t)1)
#define H5T_NATIVE_INT ((hid_t)2)
#define H5T_IEEE_F64LE ((hid_t)1)
#define H5T_STD_I32LE ((hid_t)2)

hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t file);
