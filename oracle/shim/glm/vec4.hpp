// Test infrastructure for the oracle build: forwards to the glm-compatible subset.
#pragma once
#include "fm_glm_compat.hpp"
