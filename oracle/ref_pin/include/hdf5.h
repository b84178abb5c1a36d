/* Empty stand-in: py/config.h includes <hdf5.h> for type macros that the
 * PM / COLA / 2LPT sources never expand.  TEST INFRASTRUCTURE (oracle/_ref). */
#ifndef FS2REF_HDF5_H
#define FS2REF_HDF5_H 1
#endif
