// bulk/bulk.hpp -- the whole Bulk programming interface in one include
// (same umbrella as the reference's bulk/bulk.hpp): execution policies,
// bulk::async and futures, the group heap, the agent- and group-level
// algorithms, strided_iterator and uninitialized storage.
#pragma once

#include "execution_policy.hpp"
#include "future.hpp"
#include "malloc.hpp"
#include "async.hpp"
#include "algorithm.hpp"
#include "iterator.hpp"
#include "uninitialized.hpp"
