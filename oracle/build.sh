#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure): oracle/liboracle.so from oracle/oracle.c.
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
gcc -O2 -std=c11 -fopenmp -fPIC -shared -Wall -Wextra "$here/oracle.c" -lz -o "$here/liboracle.so"
