#pragma once
#include <thrust/detail/config/compiler_fence.h>
