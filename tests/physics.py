"""Shared test configurations (physics of the reference's sample inputs)."""
PI_REF = 3.14159265358979
A0 = 5.2917720859e-11

# input/imag3d-input and input/real3d-input of the reference
G0_SAMPLE = 4. * PI_REF * 100. * 5000 * A0 / 1e-6
GD0_SAMPLE = 3. * 132.7 * 5000 * A0 / 1e-6
SAMPLE = dict(nx=128, ny=96, nz=80, dx=.2, dy=.2, dz=.2, dt=.005, gamma=.5, nu=1., lamda=1.5, cutoff=10., opt=2)


def parse_rows(path):
    """Numeric columns of the 'Initial'/'After ...' rows of an out or rms file."""
    import re
    rows = {}
    pat = re.compile(r"^\s*(Initial|After NSTP|After NPAS|After NRUN)\s*(iter\.)?\s*:(.*)$")
    for line in open(path):
        m = pat.match(line)
        if m:
            rows[m.group(1)] = [float(v) for v in m.group(3).split()]
    return rows
