// Build shim (test infrastructure): the reference's headers use std::vector,
// std::stack and std algorithms without including them; pull them in ahead
// of the system <omp.h>.
#include_next <omp.h>
#include <vector>
#include <stack>
#include <algorithm>
#include <random>
#include <string>
