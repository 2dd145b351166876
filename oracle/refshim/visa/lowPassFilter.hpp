#include "visa.hpp"
