#!/usr/bin/env bash
# Runs the reference driver (oracle/_ref/apo_ref_driver, built by oracle/ref_build.sh) on
# every input written by `make_golden.py inputs <dir>`, dumping each case to <dump_root>/<case>.
# Needs a GPU. Usage: bash tests/golden/dump_reference.sh <dir> <dump_root> [case ...]
# REF_TIMEOUT (seconds, default 300) bounds each case.
set -u
IN="$1"; OUT="$2"; shift 2
ROOT="$(cd "$(dirname "${BASH_SOURCE[0]}")/../.." && pwd)"
DRIVER="$ROOT/oracle/_ref/apo_ref_driver"
cases=("$@")
if [ ${#cases[@]} -eq 0 ]; then
    for f in "$IN"/*.f32; do cases+=("$(basename "$f" .f32)"); done
fi
rc=0
for c in "${cases[@]}"; do
    mkdir -p "$OUT/$c"
    args="$(cat "$IN/$c.args")"
    # shellcheck disable=SC2086
    timeout "${REF_TIMEOUT:-300}" "$DRIVER" "$IN/$c.f32" "$OUT/$c" $args > "$OUT/$c/log.txt" 2>&1 || { echo "failed: $c"; rc=1; }
done
exit $rc
