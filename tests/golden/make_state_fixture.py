"""Cut the particle-state fixture from the reference's resume file.

Keeps the header and every 8th particle row of the reference's
input/resume_data/particle_state_00500.csv (a 2D flow state written by the
reference solver) as tests/golden/particle_state_00500_sub8.csv, verbatim, so
the state reader is pinned on text the reference wrote and the FMM is tested
on a real particle distribution (tests/cases2d.py: "state500"). Runs here only
(it reads the reference tree); then regenerate the case's golden file with

    python tests/golden/make_golden.py state500
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: $VPM_REFERENCE_DIR, else "reference" beside the repository.
REF = os.environ.get("VPM_REFERENCE_DIR") or os.path.abspath(os.path.join(HERE, "..", "..", "..", "reference"))
SRC = os.path.join(REF, "input", "resume_data", "particle_state_00500.csv")
DST = os.path.join(HERE, "particle_state_00500_sub8.csv")
STRIDE = 8


def main():
    with open(SRC, "r", newline="") as f:
        lines = f.read().split("\n")
    header, rows = lines[0], [r for r in lines[1:] if r]
    keep = rows[::STRIDE]
    with open(DST, "w", newline="") as f:
        f.write("\n".join([header] + keep) + "\n")
    print(DST, len(keep), "of", len(rows), "rows")


if __name__ == "__main__":
    main()
