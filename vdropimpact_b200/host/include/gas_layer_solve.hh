// The model gas layer (gas_layer_solve.hh of the reference) for drivers that
// include it by that name; the class lives in gas_layer.hh with its base.
#ifndef VDI_HOST_GAS_LAYER_SOLVE_HH
#define VDI_HOST_GAS_LAYER_SOLVE_HH

#include "gas_layer.hh"

#endif
