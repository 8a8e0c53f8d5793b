/* Minimal stand-in for <netcdf.h>: the reference headers name nc_type in
 * prototypes of NetCDF helpers the tracer step never calls. */
#ifndef ORACLE_STUB_NETCDF_H
#define ORACLE_STUB_NETCDF_H
typedef int nc_type;
#define NC_NOERR 0
#define NC_GLOBAL -1
#define NC_MAX_NAME 256
#define NC_MAX_VAR_DIMS 1024
#define NC_UNLIMITED 0L
#endif
