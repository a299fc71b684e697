// host_shared.h -- force-included (after compat.h) into the group-emulation
// translation unit: shared-memory variables become static storage, which one
// group at a time owns on the host.
#pragma once
#include "compat.h"
#undef __shared__
#define __shared__ static
