// Stand-in for the absent `cth` utility library (oracle/_ref build only):
// formatting is compiled out with -DDISABLE_CPP23.
#pragma once
