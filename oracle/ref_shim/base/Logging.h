// Stand-in for the reference's base/Logging.h (which includes TensorRT's
// NvInfer.h) for compiling the reference's header-only solver math on the
// host: the size checks its solver types use, as plain asserts.
// TEST INFRASTRUCTURE.
#pragma once
#include <cassert>
#include <iostream>
#define FUNCTION_CHECK(x) assert(x)
#define FUNCTION_CHECK_EQ(x, y) assert((x) == (y))
#define FUNCTION_CHECK_NE(x, y) assert((x) != (y))
#define FUNCTION_CHECK_LT(x, y) assert((x) < (y))
#define FUNCTION_CHECK_GT(x, y) assert((x) > (y))
#define FUNCTION_CHECK_LE(x, y) assert((x) <= (y))
#define FUNCTION_CHECK_GE(x, y) assert((x) >= (y))
