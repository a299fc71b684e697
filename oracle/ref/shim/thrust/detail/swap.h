#pragma once
#include <thrust/swap.h>
