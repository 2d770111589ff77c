#!/usr/bin/env bash
# build_ref.sh -- TEST INFRASTRUCTURE ONLY: builds the reference solver itself
# (mhsuhail00/CFD_Solver s.cpp) as the parity checker and the timed CPU baseline.
#
# The reference source is read where it lies and streamed through a few literal
# substitutions straight into g++ (no copy of it is written anywhere):
#   * grid capacity np1/np2 (s.cpp:13-14) -> REF_NP1/REF_NP2 (compile time)
#   * physics members Ri, F, Pr, alpha, Re, dt and MAXSTEP (s.cpp:159-178)
#     -> read from the environment with the reference's values as defaults
#   * the two local `tol`/`maxiter` pairs of sip9p (s.cpp:2085-2086) and gauss
#     (s.cpp:2289-2290) -> CFD_TOL_SIP/CFD_MAXIT_SIP and CFD_TOL_GS/CFD_MAXIT_GS
#   * a per-step diagnostics record right after Nuss is computed (s.cpp:1982)
#   * main's second full timeLoop() (s.cpp:2450) -> a binary field dump
# See oracle/ref_hooks.h for the environment variables and the dump format.
#
# Outputs go only to oracle/_ref/ (git-ignored): cfd_ref (350x570 capacity, the
# reference's own) and cfd_ref_big (1040x1040 capacity, for 513^2 / 1025^2 grids).
#
#   oracle/build_ref.sh [--if-present]   # --if-present: exit 0 when the sources are absent
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_DIR="${CFD_REFERENCE_DIR:-/root/reference}"
SRC="$REF_DIR/s.cpp"
OUT="$HERE/_ref"
if [ ! -f "$SRC" ]; then
    if [ "${1:-}" = "--if-present" ]; then
        echo "build_ref.sh: reference source not present; oracle/_ref/cfd_ref not rebuilt" >&2
        exit 0
    fi
    echo "build_ref.sh: reference source $SRC not found (set CFD_REFERENCE_DIR)" >&2
    exit 1
fi
mkdir -p "$OUT"

transform() {
    awk '
    /static const int np1 = 350;/ { sub(/350/, "REF_NP1"); n_np1++ }
    /static const int np2 = 570;/ { sub(/570/, "REF_NP2"); n_np2++ }
    /^[ \t]*double Ri = 0\.0;/    { sub(/0\.0;/, "ref_cfg_d(\"CFD_RI\", 0.0);"); n_ri++ }
    /^[ \t]*double F = 0\.0;/     { sub(/0\.0;/, "ref_cfg_d(\"CFD_F\", 0.0);"); n_f++ }
    /^[ \t]*double Pr = 0\.71;/   { sub(/0\.71;/, "ref_cfg_d(\"CFD_PR\", 0.71);"); n_pr++ }
    /^[ \t]*double alpha = 82\.0;/ { sub(/82\.0;/, "ref_cfg_d(\"CFD_ALPHA\", 82.0);"); n_al++ }
    /^[ \t]*double Re = 1000\.0;/ { sub(/1000\.0;/, "ref_cfg_d(\"CFD_RE\", 1000.0);"); n_re++ }
    /^[ \t]*double dt = 0\.01e-2;/ { sub(/0\.01e-2;/, "ref_cfg_d(\"CFD_DT\", 0.01e-2);"); n_dt++ }
    /^[ \t]*int MAXSTEP = 5000000;/ { sub(/5000000;/, "ref_cfg_i(\"CFD_MAXSTEP\", 5000000);"); n_ms++ }
    /^[ \t]*double tol = 0\.75e-2;/ {
        n_tol++
        if (n_tol == 1) sub(/0\.75e-2;/, "ref_cfg_d(\"CFD_TOL_SIP\", 0.75e-2);")
        else            sub(/0\.75e-2;/, "ref_cfg_d(\"CFD_TOL_GS\", 0.75e-2);")
    }
    /^[ \t]*int maxiter = 100000;/ {
        n_mi++
        if (n_mi == 1) sub(/100000;/, "ref_cfg_i(\"CFD_MAXIT_SIP\", 100000);")
        else           sub(/100000;/, "ref_cfg_i(\"CFD_MAXIT_GS\", 100000);")
    }
    /^[ \t]*double Nuss = \(2 \* temp_i\)/ {
        $0 = $0 " ref_diag(loop, time, dmax, cl, cd, cm, Nuss, circ, CL_pr, CD_pr, CL_vor, CD_vor);"
        n_nu++
    }
    /^[ \t]*solver\.timeLoop\(\);/ { sub(/solver\.timeLoop\(\);/, "ref_dump(solver);"); n_main++ }
    { print }
    END {
        if (n_np1 != 1 || n_np2 != 1 || n_ri != 1 || n_f != 1 || n_pr != 1 || n_al != 1 ||
            n_re != 1 || n_dt != 1 || n_ms != 1 || n_tol != 2 || n_mi != 2 || n_nu != 1 ||
            n_main != 1) {
            print "build_ref.sh: reference source did not match the expected layout" > "/dev/stderr"
            exit 3
        }
    }' "$SRC"
}

build_one() {
    local name="$1" np1="$2" np2="$3"
    transform | g++ -O2 -ffp-contract=off -std=c++17 -w \
        -DREF_NP1="$np1" -DREF_NP2="$np2" \
        -include "$HERE/ref_hooks.h" -x c++ - -o "$OUT/$name"
}

build_one cfd_ref 350 570
build_one cfd_ref_big 1040 1040
echo "built $OUT/cfd_ref $OUT/cfd_ref_big"
