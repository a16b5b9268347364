/* Empty stand-in: the reference headers include HDF5 but the compiled parts
 * (kernels, SimParams, HSSOA sort) never use it. */
#pragma once
