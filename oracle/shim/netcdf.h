/* Empty stand-in: the reference's src/io_utils.cpp includes <netcdf.h> but
 * uses nothing from it on the hot path (test infrastructure only). */
#ifndef SBSLPM_ORACLE_SHIM_NETCDF_H
#define SBSLPM_ORACLE_SHIM_NETCDF_H
#endif
