"""GSvit's self-test decks as make_test writes them (tests.c:93-268) for the
TSF + CPML + NFFF cases: the .par file and its material vector file."""
import os


def write_deck(dirname: str, res: int, code: str, nsteps: int) -> str:
    """code "31111": electric voxel box with MATMODE_CHECK 1; "35011": PEC box."""
    mat, matcheck = code[0:2], code[2]
    ident = f"{res}{code}"
    par = os.path.join(dirname, f"{ident}.par")
    matname = f"{ident}_mat"
    lines = [f"POOL\n{res} {res} {res} 1e-6 1e-6 1e-6\n", f"COMP\n{nsteps}\n",
             f"MATMODE_CHECK\n{1 if matcheck == '1' else 0}\n", "THREADS\n4\n", f"MEDIUM_VECTOR\n{matname}\n"]
    with open(os.path.join(dirname, matname), "w") as fm:
        if mat == "31":
            fm.write(f"8 {res // 2 + 10} 30 30 {res - 30} {res - 30} {res - 30} 0 2 1 0 0\n")
        elif mat == "35":
            fm.write(f"8 {res // 2 + 10} 30 30 {res - 30} {res - 30} {res - 30} 10\n")
        else:
            raise ValueError(code)
    lines.append(f"NFFF\n16 16 16 {res - 16} {res - 16} {res - 16} 1 10000000\n\n"
                 f"NFFF_RAMAHI_POINT\n{res - 12} {res - 12} {res - 12} {ident}\n")
    lines.append(f"SOURCE_TSF\n20 20 20 {res - 20} {res - 20} {res - 20} 1.57079632679 1.57079632679 0 2 20e-6 10 5\n")
    lines.append("BOUNDARY_ALL\ncpml 10 3 -1 0.03 4\n")
    with open(par, "w") as fp:
        fp.write("\n".join(lines) + "\n")
    return par
