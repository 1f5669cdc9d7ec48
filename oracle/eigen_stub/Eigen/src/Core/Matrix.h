// Minimal Eigen-API stand-in (see Eigen/Core), for sources that include this
// internal header directly.
#include "../../Core"
