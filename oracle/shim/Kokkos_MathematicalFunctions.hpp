// Forwarding header: see kokkos_ekat_shim.hpp (test infrastructure only).
#pragma once
#include "kokkos_ekat_shim.hpp"
