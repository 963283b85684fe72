// glm-subset shim entry header (project-written; see shim_core.hpp).
#pragma once
#include "shim_core.hpp"
