#pragma once
#include "tarch/la/Scalar.h"
