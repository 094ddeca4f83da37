"""CPU oracle of the dpa advection path (test infrastructure: the checker and
the timed CPU baseline). See oracle.cpp for the restated reference functions."""
