/* Stand-in for HDF5's H5Tpublic.h: everything lives in the shim hdf5.h. */
#include "hdf5.h"
