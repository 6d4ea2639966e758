// Fused pipeline stages: declarations live in the public C ABI header.
#pragma once
#include "../../include/alenka_b200.h"
