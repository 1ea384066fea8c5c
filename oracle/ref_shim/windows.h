/* Linux stand-in for <windows.h> (included by the reference's Console.h:5).
 * The reference relies on windows.h bringing min/max into scope (PI.h:97,105). */
#pragma once
#include <algorithm>
using std::max;
using std::min;
