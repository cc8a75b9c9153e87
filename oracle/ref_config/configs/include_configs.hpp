#include "configs/reference/config.hpp"
#include "configs/haswell/config.hpp"
#include "configs/zen/config.hpp"
