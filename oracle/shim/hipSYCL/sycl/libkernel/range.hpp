// Forwarding header of the host oracle shim (test infrastructure).
#pragma once
#include <sycl/sycl.hpp>
