#!/bin/sh
# TEST INFRASTRUCTURE: builds the CPU emulation of libclarity (the library's
# own kernel and host sources compiled as C++ with AddressSanitizer) into
# _build/emu/emu_main.  Usage: tests/emu/build_emu.sh [repo root]
set -e
ROOT=${1:-$(cd "$(dirname "$0")/../.." && pwd)}
OUT="$ROOT/_build/emu"
mkdir -p "$OUT"
CXX=${EMU_CXX:-/usr/bin/g++}
FLAGS="-std=c++20 -O1 -g -fsanitize=address -fno-omit-frame-pointer -DCLARITY_HOST_EMULATION \
 -I$ROOT/tests/emu -I$ROOT/clarity_b200/csrc -I/usr/local/cuda/include"
pids=""
for f in "$ROOT"/clarity_b200/csrc/*.cu "$ROOT"/clarity_b200/csrc/*.cpp \
         "$ROOT"/tests/emu/emu_runtime.cpp "$ROOT"/tests/emu/emu_main.cpp; do
  $CXX $FLAGS -x c++ -c "$f" -o "$OUT/$(basename "$f").o" &
  pids="$pids $!"
done
for p in $pids; do wait $p; done
$CXX -fsanitize=address "$OUT"/*.o -o "$OUT/emu_main"
