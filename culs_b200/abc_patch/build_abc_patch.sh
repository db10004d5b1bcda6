#!/bin/sh
# Builds `abcg`: ABC with the GPU commands of culs_abc_patch.cpp, linked
# against libculs_b200.so.  Needs an ABC source tree that has been built with
# its own Makefile (libabc.a in its root): CULS_ABC_ROOT=/path/to/abc.
#
#   CULS_ABC_ROOT=/path/to/abc sh culs_b200/abc_patch/build_abc_patch.sh
#
# Without CULS_ABC_ROOT it does nothing and says so.
set -eu
if [ -z "${CULS_ABC_ROOT:-}" ]; then
    echo "CULS_ABC_ROOT is not set: the ABC front end is not built" >&2
    exit 0
fi
HERE=$(cd "$(dirname "$0")" && pwd)
PKG=$(dirname "$HERE")
ROOT=$(dirname "$PKG")
ABC="$CULS_ABC_ROOT"
# the platform defines ABC's own Makefile passes
DEFS="-DLIN64 -DSIZEOF_VOID_P=8 -DSIZEOF_LONG=8 -DSIZEOF_INT=4 -DABC_USE_STDINT_H=1"
g++ -O2 -std=c++17 -fPIC $DEFS -I "$ABC/src" -I "$ROOT/include" -I "$HERE" \
    -c "$HERE/culs_abc_patch.cpp" -o "$PKG/abc_patch.o"
# ABC's main() is src/base/main/main.o, which libabc.a leaves out
g++ -o "$PKG/abcg" "$PKG/abc_patch.o" "$ABC/src/base/main/main.o" "$ABC/libabc.a" \
    -L "$PKG" -lculs_b200 -Wl,-rpath,"$PKG" -lm -ldl -lpthread -lreadline
echo "built $PKG/abcg"
