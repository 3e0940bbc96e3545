"""Driver shared by the locally adaptive KDEs: ``fit()`` and the checkpoint keys.

The public contract kept from lakde/kdes.py:34 is the ``fit(X, iterations,
callbacks, sparsity_threshold, dataset_label)`` signature, the meaning of an
iteration (one update of every kernel) and the ``block_size`` /
``verbose`` / ``iter_steps`` state-dict keys (lakde/kdes.py:114-126).  The
driver itself is written for the two schedules of this package:

* block schedule (``fused=False``): an iteration is ``num_blocks`` kernel-block
  updates, each a ``partial_step_`` through the sm_100a library;
* fused schedule (``fused=True``): the whole kernel set is one block, so an
  iteration is one engine step, replayed from a CUDA graph once captured.

``iter_steps`` counts block updates across calls, so a model restored with
``load_state_dict`` resumes where it stopped.  Callbacks are plain callables
``cb(X, model, update_index)`` run after every update; they may raise
``StopIteration`` to end the fit early.  Device-side failures (a matrix no
jitter rung repairs, a bounded tensor-core wait that ran out) are collected
on the device and raised once at the end of ``fit`` by ``check_errors_``.
"""

from abc import ABC, abstractmethod

import torch


class VIModel(ABC):
    """Common state and the update loop of the variational KDE models."""

    def __init__(self, block_size, verbose, logs):
        self.block_size = block_size
        self.verbose = verbose
        self.iter_steps = 0
        # `logs`: any truthy value keeps the ELBO after every update in
        # `elbo_trace` (host floats; costs one device synchronisation per update)
        self.elbo_trace = [] if logs else None

    # -------------------------------------------------------- model interface
    @abstractmethod
    def init_parameters_(self, X, sparsity_threshold=None):
        """Hyper-parameters, kNN graph and initial responsibilities."""

    @abstractmethod
    def init_summaries_(self, X, sparsity_threshold=None):
        """Initial posterior summaries and normalisers."""

    @abstractmethod
    def partial_step_(self, X, block_idx, sparsity_threshold=None):
        """One update of kernel block `block_idx`."""

    @abstractmethod
    def compute_elbo(self, X):
        """Evidence lower bound of the current variational posterior."""

    @abstractmethod
    def log_pred_density(self, X, Y):
        """Predictive log density of the rows of Y."""

    @abstractmethod
    def data_log_likelihood_no_rnm(self, X):
        pass

    @abstractmethod
    def data_log_likelihood(self, X):
        pass

    def resume_(self, X, sparsity_threshold=None):
        """Prepares a model restored by ``load_state_dict`` to continue fitting
        (the models override it; nothing to do by default)."""

    def num_blocks(self, N):
        return (N - 1) // self.block_size + 1

    def check_errors_(self):
        """Raises deferred device-side failures (the models override it)."""

    # ------------------------------------------------------------------ fit
    def fit(self, X, iterations=200, callbacks=None, sparsity_threshold=None, dataset_label=None):
        if not X.is_contiguous():
            raise ValueError("Training data must be contiguous, call .contiguous() before fitting")
        threshold = sparsity_threshold or 0
        if callbacks is None:
            hooks = ()
        elif isinstance(callbacks, (list, tuple)):
            hooks = tuple(callbacks)
        else:
            hooks = (callbacks,)
        if self.iter_steps == 0:
            self.init_parameters_(X, threshold)
            self.init_summaries_(X, threshold)
        else:
            self.resume_(X, threshold)
        blocks = self.num_blocks(X.size(0))
        try:
            for _ in range(iterations * blocks):
                done = self.iter_steps
                self.partial_step_(X, done % blocks, sparsity_threshold=threshold)
                self.iter_steps = done + 1
                for hook in hooks:
                    hook(X, self, done)
                if self.verbose or self.elbo_trace is not None:
                    self._record_update(X, done, blocks)
        except (KeyboardInterrupt, StopIteration):
            pass
        self.check_errors_()
        return self

    def _record_update(self, X, done, blocks):
        elbo = float(self.compute_elbo(X))
        if self.elbo_trace is not None:
            self.elbo_trace.append(elbo)
        if self.verbose:
            print(f"update {done + 1} (iteration {done // blocks + 1}, block {done % blocks + 1}/{blocks}): "
                  f"ELBO {elbo:.6f}")

    # ---------------------------------------------------------------- outputs
    def data_likelihood(self, X):
        return torch.exp_(self.data_log_likelihood(X))

    def pred_density(self, X, Y):
        return torch.exp_(self.log_pred_density(X, Y))

    # ------------------------------------------------------------- checkpoint
    def state_dict(self):
        return {"block_size": self.block_size, "verbose": self.verbose, "iter_steps": self.iter_steps}

    def load_state_dict(self, state_dict):
        self.block_size = state_dict["block_size"]
        self.verbose = state_dict["verbose"]
        self.iter_steps = state_dict["iter_steps"]

    def hparam_state_dict(self):
        return {"block_size": self.block_size}

    def save(self, fname, state_dict=None):
        d = self.state_dict()
        if state_dict:
            d.update(state_dict)
        torch.save(d, fname)
