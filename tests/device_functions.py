"""CUDA C device functions of the device-function tests: the same formulas as the reference
harness's host callbacks (oracle/ref_harness.c: bc_moving_wall, bc_unsteady_inflow,
src_unsteady), written in teal's Compute argument order."""

MOVING_WALL = """
__device__ void lid_wall(double *out, const double *property, const double *center, double time,
                         const double *inner)
{
    // a wall moving with speed 1 along x (run/lid_driven_cavity/run.c:7-17)
    out[0] = inner[0];
    out[1] = (2 * 1.0) - inner[1];
    out[2] = -inner[2];
    out[3] = -inner[3];
    out[4] = inner[4];
}
"""

UNSTEADY_INFLOW = """
__device__ void unsteady_inflow(double *out, const double *property, const double *center, double time,
                                const double *inner)
{
    out[0] = 1 + (0.1 * sin(center[0] - time));
    out[1] = 0.5 + (0.05 * cos(center[1] + (2 * time)));
    out[2] = 0.01 * center[2];
    out[3] = 0;
    out[4] = (1 / property[0]) + (0.02 * sin(3 * time));
}
"""

UNSTEADY_SOURCE = """
__device__ void unsteady_source(double *source, const double *property, const double *center, double time,
                                const double *state)
{
    double fx = 0.1 * state[0] * sin(center[0] + time);
    double fy = 0.05 * state[0] * cos(center[1] - time);
    source[0] = 0;
    source[1] = fx;
    source[2] = fy;
    source[3] = 0;
    source[4] = (state[1] * fx) + (state[2] * fy);
}
"""



def hill_forcing(name="hill_forcing", tau="0.001"):
    """The periodic hill's forcing (run/periodic_hill/run.c:13-21: target bulk velocity 1, time
    scale 0.001) with its Prepare, the volume average of the state, read from context[5..9]."""
    return """
__device__ void NAME(double *source, const double *property, const double *center, double time,
                     const double *context)
{
    const double *state = context, *average = context + 5;
    double s1 = state[0] * (1.0 - average[1]) / TAU;
    source[1] = s1;
    source[4] = state[1] * s1;
}
""".replace("NAME", name).replace("TAU", tau)


HILL_FORCING = hill_forcing()

# writes the context's average slots into the source, to show what a source without Prepare sees
AVERAGE_PROBE = """
__device__ void average_probe(double *source, const double *property, const double *center, double time,
                              const double *context)
{
    for (int k = 0; k < 5; k++) source[k] = context[5 + k];
}
"""
