// Stand-in for the absent `cth` utility library (oracle/_ref build only): the
// hot-path headers include it but use none of its macros.
#pragma once
