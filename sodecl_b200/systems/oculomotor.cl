/*
 * Oculomotor (saccadic eye-movement) model: 6 states, 6 parameters,
 * optionally 2 noise processes.  A SODECL system file: it defines the
 * right-hand side `sode_system`, the analytic Jacobian `calc_jacobian`
 * (needed by the implicit solvers) and the diffusion term
 * `sode_system_stoch` (needed by Euler-Maruyama).
 *
 * State y = [g, u, n, r, l, m]:
 *   g  eye position            u  eye velocity
 *   n  neural integrator       r  right burst neuron
 *   l  left burst neuron       m  motor error
 * Parameters p = [alpha, beta, tau, gamma, alpha_t, beta_t] of the burst
 * non-linearity (nominal 120, 1.5, 0.0045, 0.05, 600, 9), followed by the
 * noise amplitudes when noise processes are used.
 *
 * Same model and the same floating-point evaluation order as the
 * reference's examples/oculomotor.cl (sburstf :5-20, dsburstf :22-36,
 * calc_jacobian :38-81, sode_system :83-97, sode_system_stoch :99-112),
 * so trajectories agree with the reference to the last bits.  Three
 * differences, none of which changes a trajectory: ocm_burst selects its exp
 * argument instead of branching (same values, see there); jac[4][5] carries the
 * chain-rule sign the reference's calc_jacobian omits (entries off the three
 * bands are never read by the implicit solvers), and calc_jacobian_params
 * (df/dp) and calc_vjp (the vector-Jacobian product), both for the adjoint,
 * are additions.
 */

#define OCM_T1 0.15
#define OCM_T2 0.012
#define OCM_TN 25.00
/* plant gains, folded at compile time */
#define OCM_VEL_GAIN ((1.00 / OCM_T1) + (1.00 / OCM_T2))
#define OCM_POS_GAIN (1.00 / (OCM_T1 * OCM_T2))

/* burst-neuron firing-rate non-linearity:
 *   x > 0:  at * (1 - exp(-x / bt))
 *   else:   -(a / b) * x * exp(x / b)
 * written with one exp whose argument is selected: x / (-bt) rounds exactly
 * as (-x) / bt, so each branch's value is the same to the last bit, and the
 * orbits of a warp on either side of x = 0 share one exp instead of running
 * both branches one after the other.  The argument selects between two
 * quotients, not between two divisors: bt and b are fixed for an orbit, so
 * where the compiler computes quotients through reciprocals it takes both
 * reciprocals once, outside the step loop */
double ocm_burst(double x, double a, double b, double at, double bt)
{
	int right = x > 0;
	double e = exp(right ? x / -bt : x / b);
	return right ? (at * (1.00 - e)) : (-(a / b) * x * e);
}

/* d(ocm_burst)/dx */
double ocm_burst_slope(double x, double a, double b, double at, double bt)
{
	double slope = 0;
	if (x > 0)
	{
		slope = (at * exp(-x / bt)) / bt;
	}
	else
	{
		slope = -((a * exp(x / b)) / b + (a * x * exp(x / b)) / (b * b));
	}
	return slope;
}

void sode_system(double t, double y[_numeq_], double yout[_numeq_], double p[_numpar_])
{
	double drive = y[3] - y[4];
	yout[0] = y[1];
	yout[1] = -(OCM_VEL_GAIN * y[1]) - (OCM_POS_GAIN * y[0]) + (OCM_POS_GAIN * y[2]) + OCM_VEL_GAIN * drive;
	yout[2] = -(y[2] / OCM_TN) + drive;
	yout[3] = (1.00 / p[2]) * (-y[3] - (p[3] * y[3] * y[4] * y[4]) + ocm_burst(y[5], p[0], p[1], p[4], p[5]));
	yout[4] = (1.00 / p[2]) * (-y[4] - (p[3] * y[4] * y[3] * y[3]) + ocm_burst(-y[5], p[0], p[1], p[4], p[5]));
	yout[5] = -drive;
}

void calc_jacobian(double y[_numeq_], double jac[_numeq_][_numeq_], double p[_numpar_])
{
	int i, j;
	for (i = 0; i < 6; i++)
	{
		for (j = 0; j < 6; j++)
		{
			jac[i][j] = 0;
		}
	}
	jac[0][1] = 1;

	jac[1][0] = -1 / (OCM_T1 * OCM_T2);
	jac[1][1] = -(1 / OCM_T1) - (1 / OCM_T2);
	jac[1][2] = 1 / (OCM_T1 * OCM_T2);
	jac[1][3] = (1 / OCM_T1) + (1 / OCM_T2);
	jac[1][4] = -(1 / OCM_T1) - (1 / OCM_T2);

	jac[2][2] = -1 / OCM_TN;
	jac[2][3] = 1;
	jac[2][4] = -1;

	jac[3][3] = -(p[3] * (y[4] * y[4]) + 1) / p[2];
	jac[3][4] = -(2 * p[3] * y[4] * y[3]) / p[2];
	jac[3][5] = ocm_burst_slope(y[5], p[0], p[1], p[4], p[5]) / p[2];

	jac[4][3] = -(2 * p[3] * y[4] * y[3]) / p[2];
	jac[4][4] = -(p[3] * (y[3] * y[3]) + 1) / p[2];
	/* d/dy5 of ocm_burst(-y5): note the chain-rule sign, which the reference's
	 * file omits (its banded solve never reads this entry, so the solvers'
	 * results are the same either way; full-Jacobian users need the sign) */
	jac[4][5] = -ocm_burst_slope(-y[5], p[0], p[1], p[4], p[5]) / p[2];

	jac[5][3] = -1;
	jac[5][4] = 1;
}

/* ocm_burst(x, ...) and its derivatives d[0..3] w.r.t. (a, b, at, bt), with
 * one exp (argument selected as in ocm_burst) */
double ocm_burst_dparams(double x, double a, double b, double at, double bt, double d[4])
{
	int right = x > 0;
	double e = exp(x / (right ? -bt : b));
	double ib = 1.00 / b;
	double ibt = 1.00 / bt;
	d[0] = right ? (double)0 : -(x * e) * ib;
	d[1] = right ? (double)0 : (a * x * e) * ib * ib * (1.00 + x * ib);
	d[2] = right ? 1.00 - e : (double)0;
	d[3] = right ? -(at * x * e) * ibt * ibt : (double)0;
	return right ? (at * (1.00 - e)) : (-(a * ib) * x * e);
}

/* df/dp, jacp[i][k] = d yout[i] / d p[k] for the six model parameters.  Not in
 * the reference's file: the adjoint (model fitting) uses it together with
 * calc_jacobian; without it the adjoint differentiates sode_system itself.
 * Only gradients depend on it, so it shares subexpressions freely (one exp per
 * burst, one reciprocal of tau). */
void calc_jacobian_params(double y[_numeq_], double jacp[_numeq_][_numpar_], double p[_numpar_])
{
	int i, k;
	double dr[4], dl[4];
	for (i = 0; i < 6; i++)
	{
		for (k = 0; k < _numpar_; k++)
		{
			jacp[i][k] = 0;
		}
	}
	double itau = 1.00 / p[2];
	double br = ocm_burst_dparams(y[5], p[0], p[1], p[4], p[5], dr);
	double bl = ocm_burst_dparams(-y[5], p[0], p[1], p[4], p[5], dl);
	double r = -y[3] - (p[3] * y[3] * y[4] * y[4]) + br;
	double l = -y[4] - (p[3] * y[4] * y[3] * y[3]) + bl;
	jacp[3][0] = dr[0] * itau;
	jacp[3][1] = dr[1] * itau;
	jacp[3][2] = -r * itau * itau;
	jacp[3][3] = -(y[3] * y[4] * y[4]) * itau;
	jacp[3][4] = dr[2] * itau;
	jacp[3][5] = dr[3] * itau;
	jacp[4][0] = dl[0] * itau;
	jacp[4][1] = dl[1] * itau;
	jacp[4][2] = -l * itau * itau;
	jacp[4][3] = -(y[4] * y[3] * y[3]) * itau;
	jacp[4][4] = dl[2] * itau;
	jacp[4][5] = dl[3] * itau;
}

/* ocm_burst and its slope and parameter derivatives with one exp:
 * d = [dB/dx, dB/da, dB/db, dB/dat, dB/dbt] */
double ocm_burst_all(double x, double a, double b, double at, double bt, double d[5])
{
	int right = x > 0;
	double e = exp(x / (right ? -bt : b));
	double ib = 1.00 / b;
	double ibt = 1.00 / bt;
	double g = 1.00 + x * ib;
	d[0] = right ? at * e * ibt : -(a * ib) * e * g;
	d[1] = right ? (double)0 : -(x * e) * ib;
	d[2] = right ? (double)0 : (a * x * e) * ib * ib * g;
	d[3] = right ? 1.00 - e : (double)0;
	d[4] = right ? -(at * x * e) * ibt * ibt : (double)0;
	return right ? (at * (1.00 - e)) : (-(a * ib) * x * e);
}

/* ybar[j] += sum_i v[i] d yout[i] / d y[j], pbar[k] += sum_i v[i] d yout[i] / d p[k]
 * for the six model parameters: the vector-Jacobian product of sode_system,
 * term by term (not in the reference's file; the adjoint uses it in place of
 * calc_jacobian and calc_jacobian_params) */
void calc_vjp(double t, double y[_numeq_], double v[_numeq_], double ybar[_numeq_], double pbar[_numpar_],
              double p[_numpar_])
{
	double itau = 1.00 / p[2];
	double dr[5], dl[5];
	double br = ocm_burst_all(y[5], p[0], p[1], p[4], p[5], dr);
	double bl = ocm_burst_all(-y[5], p[0], p[1], p[4], p[5], dl);
	double wr = v[3] * itau;
	double wl = v[4] * itau;
	/* drive = y3 - y4 enters yout1 (gain VEL), yout2 (1) and yout5 (-1) */
	double vdrive = v[1] * OCM_VEL_GAIN + v[2] - v[5];
	ybar[0] += -(v[1] * OCM_POS_GAIN);
	ybar[1] += v[0] - v[1] * OCM_VEL_GAIN;
	ybar[2] += v[1] * OCM_POS_GAIN - v[2] / OCM_TN;
	ybar[3] += vdrive + wr * (-1.00 - p[3] * y[4] * y[4]) + wl * (-2.00 * p[3] * y[4] * y[3]);
	ybar[4] += -vdrive + wr * (-2.00 * p[3] * y[3] * y[4]) + wl * (-1.00 - p[3] * y[3] * y[3]);
	ybar[5] += wr * dr[0] - wl * dl[0];
	double r = -y[3] - (p[3] * y[3] * y[4] * y[4]) + br;
	double l = -y[4] - (p[3] * y[4] * y[3] * y[3]) + bl;
	pbar[0] += wr * dr[1] + wl * dl[1];
	pbar[1] += wr * dr[2] + wl * dl[2];
	pbar[2] += -(wr * r + wl * l) * itau;
	pbar[3] += -(wr * y[3] * y[4] * y[4] + wl * y[4] * y[3] * y[3]);
	pbar[4] += wr * dr[3] + wl * dl[3];
	pbar[5] += wr * dr[4] + wl * dl[4];
}

void sode_system_stoch(double t, double y[_numeq_], double stoch[_numeq_], double p[_numpar_], double noise[_numnoi_])
{
	int k;
	for (k = 0; k < 6; k++)
	{
		stoch[k] = 0;
	}
	stoch[1] = OCM_VEL_GAIN * (y[3] - y[4]) * p[_numpar_ - _numnoi_ + 0] * noise[0] + p[_numpar_ - _numnoi_ + 1] * noise[1];
}
