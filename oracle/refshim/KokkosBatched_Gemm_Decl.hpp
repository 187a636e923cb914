// TEST INFRASTRUCTURE ONLY: see KokkosBatched_Gemv_Decl.hpp
#include "KokkosBatched_Gemv_Decl.hpp"
