"""numpy implementations of the analysis steps of adamantine_b200.sharded --
test infrastructure: they let the multi-process exchange run on CPU ranks
(gloo) and be checked against the single-process restatement."""
import numpy as np
import torch


class NumpySteps:
    """loc: None, or (rho_obs (m, m), rho_state (n_state, m)) -- the
    localization weights between observations and between state entries and
    observations; gain keeps HA and Z for the localized partial update."""

    def __init__(self, loc=None):
        self.loc = loc
        self.HA = self.Z = None

    def observe(self, states, n_state, obs_index):
        X = states.numpy()
        idx = obs_index.numpy()
        return torch.from_numpy(np.stack([X[k, idx[k]] for k in range(X.shape[0])]))

    def gain(self, hx, obs, perturbations, obs_var=None, obs_cov=None):
        HX = hx.numpy()
        N = HX.shape[0]
        HA = HX - HX.mean(axis=0)
        R = np.diag(obs_var.numpy()) if obs_cov is None else obs_cov.numpy()
        B = HA.T @ HA / (N - 1.0)
        if self.loc is not None:
            B = B * self.loc[0]
        C = B + R
        D = obs.numpy()[None, :] + perturbations.numpy() - HX
        Z = np.linalg.solve(C, D.T)
        self.HA, self.Z = HA, Z
        return torch.from_numpy(HA @ Z / (N - 1.0))

    def local_sum(self, states, n_state, params):
        s = states.numpy()[:, :n_state].sum(axis=0)
        if params is not None:
            s = np.concatenate([s, params.numpy().sum(axis=0)])
        return torch.from_numpy(s)

    def partial_update(self, states, n_state, params, total, w_rows, first=0):
        X = states.numpy()[:, :n_state]
        if params is not None:
            X = np.concatenate([X, params.numpy()], axis=1)
        N = w_rows.shape[1]
        A = X - total.numpy()[None, :] / N
        U = w_rows.numpy().T @ A
        if self.loc is not None:
            # state rows: sum_j rho_ij (sum_k local A_k[i] HA_k[j]) Z[j][l] / (N - 1)
            n_local = A.shape[0]
            G = A[:, :n_state].T @ self.HA[first:first + n_local] / (N - 1.0)  # (n_state, m)
            U[:, :n_state] = ((G * self.loc[1]) @ self.Z).T
        return torch.from_numpy(U)

    def apply(self, states, n_state, params, u, update_mask=None):
        U = u.numpy()
        upd = U[:, :n_state]
        if update_mask is not None:
            upd = upd * (update_mask.numpy() != 0)
        states[:, :n_state] += torch.from_numpy(upd)
        if params is not None:
            params += torch.from_numpy(U[:, n_state:])
