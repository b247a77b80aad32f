// Oracle test infrastructure: boost::make_shared as std::make_shared.
#pragma once
#include <memory>
namespace boost { using std::make_shared; }
