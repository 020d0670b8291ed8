/* NetCDF type constants used by the reference's headers.  TEST
 * INFRASTRUCTURE (oracle/ref): no NetCDF I/O is compiled into the driver. */
#ifndef CGFD_REF_STUB_NETCDF_H
#define CGFD_REF_STUB_NETCDF_H
#define NC_INT 4
#define NC_FLOAT 5
#define NC_DOUBLE 6
#define NF4FLOAT 9.9692099683868690e+36f
#define NF4DOUBLE 9.9692099683868690e+36
#endif
