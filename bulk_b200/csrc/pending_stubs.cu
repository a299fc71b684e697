#include "bk_common.cuh"
namespace bk {
}
