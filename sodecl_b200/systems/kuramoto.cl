/*
 * Kuramoto model of N = _numeq_ coupled phase oscillators:
 *
 *   d(theta_i)/dt = omega_i + (K/N) * sum_j sin(theta_j - theta_i)
 *
 * with the sum over every j, i included.  Parameters p = [K, omega_1..N],
 * followed by N noise amplitudes sigma_1..N when the system is integrated
 * with Euler-Maruyama (additive noise sigma_i * dW_i).
 *
 * `sode_system` and `sode_system_stoch` evaluate in the same floating-point
 * order as the reference's examples/kuramoto.cl (:3-16, :18-24).
 * The reference ships no Jacobian for this model; `calc_jacobian` below is
 * this library's addition so the implicit solvers can integrate it:
 *   J_ij = (K/N) cos(theta_j - theta_i)               (j != i)
 *   J_ii = -(K/N) sum_{j != i} cos(theta_j - theta_i)
 * `sode_system_row`, `sode_system_stoch_row` and `calc_jacobian_band` (also
 * additions) give one equation's terms and its row's three band entries
 * (columns i-1, i, i+1), evaluated exactly as `sode_system`,
 * `sode_system_stoch` and `calc_jacobian` evaluate them; with them, several
 * lanes of a warp can share one orbit (lanes per orbit).
 * `sode_system_row_band` gives a row's right-hand side and band together.
 */

void sode_system(double t, double y[_numeq_], double yout[_numeq_], double p[_numpar_])
{
	for (int i = 0; i < _numeq_; i++)
	{
		double coupling = 0;
		for (int j = 0; j < _numeq_; j++)
		{
			coupling = coupling + (sin(y[j] - y[i]));
		}
		coupling = coupling * (double)(p[0] / (double)(_numeq_));
		yout[i] = coupling + p[i + 1];
	}
}

double sode_system_row(int i, double t, double y[_numeq_], double p[_numpar_])
{
	double coupling = 0;
	for (int j = 0; j < _numeq_; j++)
	{
		coupling = coupling + (sin(y[j] - y[i]));
	}
	coupling = coupling * (double)(p[0] / (double)(_numeq_));
	return coupling + p[i + 1];
}

void calc_jacobian(double y[_numeq_], double jac[_numeq_][_numeq_], double p[_numpar_])
{
	double scale = (double)(p[0] / (double)(_numeq_));
	for (int i = 0; i < _numeq_; i++)
	{
		double diag = 0;
		for (int j = 0; j < _numeq_; j++)
		{
			double c = scale * cos(y[j] - y[i]);
			jac[i][j] = c;
			if (j != i)
			{
				diag = diag - c;
			}
		}
		jac[i][i] = diag;
	}
}

void calc_jacobian_band(int i, double y[_numeq_], double band[3], double p[_numpar_])
{
	double scale = (double)(p[0] / (double)(_numeq_));
	double diag = 0;
	band[0] = 0;
	band[2] = 0;
	for (int j = 0; j < _numeq_; j++)
	{
		double c = scale * cos(y[j] - y[i]);
		if (j == i - 1)
		{
			band[0] = c;
		}
		if (j == i + 1)
		{
			band[2] = c;
		}
		if (j != i)
		{
			diag = diag - c;
		}
	}
	band[1] = diag;
}

/* sode_system_row and calc_jacobian_band of row i in one evaluation, with
 * sin and cos of each difference from one sincos: returns yout[i], fills
 * band[0..2] (columns i-1, i, i+1); both are the same values those two
 * functions give.  The implicit solvers with lanes per orbit use it (each
 * Newton pass needs the row and, until it converges, the band at the same
 * point). */
double sode_system_row_band(int i, double t, double y[_numeq_], double band[3], double p[_numpar_])
{
	double scale = (double)(p[0] / (double)(_numeq_));
	double coupling = 0;
	double diag = 0;
	band[0] = 0;
	band[2] = 0;
	for (int j = 0; j < _numeq_; j++)
	{
		double cosine;
		double sine = sincos(y[j] - y[i], &cosine);
		coupling = coupling + sine;
		double c = scale * cosine;
		if (j == i - 1)
		{
			band[0] = c;
		}
		if (j == i + 1)
		{
			band[2] = c;
		}
		if (j != i)
		{
			diag = diag - c;
		}
	}
	band[1] = diag;
	coupling = coupling * (double)(p[0] / (double)(_numeq_));
	return coupling + p[i + 1];
}

void sode_system_stoch(double t, double y[_numeq_], double stoch[_numeq_], double p[_numpar_], double noise[_numnoi_])
{
	for (int i = 0; i < _numeq_; i++)
	{
		stoch[i] = p[_numpar_ - _numnoi_ + i] * noise[i];
	}
}

double sode_system_stoch_row(int i, double t, double y[_numeq_], double p[_numpar_], double noise[_numnoi_])
{
	return p[_numpar_ - _numnoi_ + i] * noise[i];
}
