// Project-written empty stand-in (TEST INFRASTRUCTURE ONLY): dynex.cc includes it but uses nothing from it.
#pragma once
#include <array>
