/* Serial stand-in for Peano's pfor: the harness parallelises over cells. */
#pragma once
#define pfor(counter, from, to, grain) for (int counter = (from); counter < (to); counter++) {
#define endpfor }
