/* Oracle shim: see serialization.hpp. */
#pragma once
#include <boost/serialization/serialization.hpp>
