#pragma once
#ifndef DIMENSIONS
#error DIMENSIONS must be defined
#endif
