#pragma once
#include "pxr/base/gf/gf_shim.h"
