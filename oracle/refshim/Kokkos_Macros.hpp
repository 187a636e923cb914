// TEST INFRASTRUCTURE ONLY: see Kokkos_Core.hpp
#include "Kokkos_Core.hpp"
