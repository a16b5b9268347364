/* Stand-in for <H5Cpp.h>.  The reference headers include HDF5 but the
 * compiled parts (kernels, SimParams, HSSOA sort, PrepareFrameArrays) never
 * call it; snapshotmanager.h only names H5::H5File in declarations. */
#pragma once
namespace H5 { class H5File; }
