#pragma once
#include <cstddef>
#include "access.hpp"
