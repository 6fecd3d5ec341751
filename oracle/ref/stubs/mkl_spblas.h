// The reference includes both MKL headers; every declaration it needs is in mkl.h.
#pragma once
#include "mkl.h"
