// Stand-in for the reference's base/Constants.h (run configuration, which
// pulls in OpenCV through its config parser). The image-term header that
// includes it uses none of its constants. TEST INFRASTRUCTURE.
#pragma once
#include <base/CommonTypes.h>
