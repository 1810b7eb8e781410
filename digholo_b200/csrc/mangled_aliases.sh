#!/bin/sh
# Writes a linker script that exports every reference entry point declared
# in include/digHolo.h also under its C++-mangled name (the names the
# reference's Linux build exports, its EXT_C being empty there), as an
# alias of the C-linkage function: "_Z13digHoloCreatev = digHoloCreate;".
# The mangled names come from g++ itself: a generated C++ file takes the
# address of each function declared with C++ linkage.
# usage: mangled_aliases.sh <include dir> <output .ld>
set -e
INC="$1"
OUT="$2"
DIR=$(dirname "$OUT")
NAMES=$(sed -n 's/^[A-Za-z_][A-Za-z0-9_ *]*[ *]\(digHolo[A-Za-z0-9_]*\)(.*/\1/p' "$INC/digHolo.h" | grep -v '^digHoloB200' | sort -u)
SRC="$DIR/mangled_refs.cpp"
{
    echo '#define DIGHOLO_CXX_LINKAGE'
    echo '#include "digHolo.h"'
    echo 'void* const dh_mangled_refs[] = {'
    for n in $NAMES; do echo "    (void*)&$n,"; done
    echo '};'
} > "$SRC"
g++ -std=c++11 -c -I"$INC" "$SRC" -o "$DIR/mangled_refs.o"
: > "$OUT"
for m in $(nm -u "$DIR/mangled_refs.o" | awk '{print $2}' | grep '^_Z'); do
    plain=$(echo "$m" | c++filt | sed 's/(.*//')
    echo "$m = $plain;" >> "$OUT"
done
test -s "$OUT"
