#pragma once
#include "boost/serialization/wk_stub_serialization.hpp"
