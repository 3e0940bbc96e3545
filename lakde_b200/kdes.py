"""Model API shell: the fit loop, callbacks and state dict (lakde/kdes.py:8-135)."""

from abc import ABC, abstractmethod

import torch

from .callbacks import ELBOCallback


class AbstractKDE(ABC):
    def __init__(self, block_size, verbose, logs):
        self.block_size = block_size
        self.verbose = verbose
        self.iter_steps = 0
        self.logger = None
        if logs:
            from torch.utils.tensorboard import SummaryWriter

            self.logger = SummaryWriter(log_dir=logs) if isinstance(logs, str) else SummaryWriter()

    @abstractmethod
    def init_parameters_(self, X, sparsity_threshold=None):
        pass

    @abstractmethod
    def init_summaries_(self, X, sparsity_threshold=None):
        pass

    @abstractmethod
    def partial_step_(self, X, block_idx, sparsity_threshold=None):
        pass

    def num_blocks(self, N):
        return (N - 1) // self.block_size + 1

    def fit(self, X, iterations=200, callbacks=None, sparsity_threshold=None, dataset_label=None):
        """Initialise once, then run `iterations` passes over all kernel blocks
        (lakde/kdes.py:34-87).  KeyboardInterrupt and StopIteration end the fit."""
        N, D = X.shape
        assert X.is_contiguous(), "Training data must be contiguous, call .contiguous() before fitting"
        if sparsity_threshold is None:
            sparsity_threshold = 0
        if callbacks is None:
            callbacks = ELBOCallback(verbose=self.verbose)
        if self.iter_steps < 1:
            if self.verbose:
                print("Initializing parameters...")
            self.init_parameters_(X, sparsity_threshold)
            self.init_summaries_(X, sparsity_threshold)
        num_blocks = self.num_blocks(N)
        if self.verbose:
            print("Fitting data...")
        try:
            for _ in range(iterations):
                epoch = self.iter_steps // num_blocks
                for bi in range(num_blocks):
                    self.partial_step_(X, bi, sparsity_threshold=sparsity_threshold)
                    if self.verbose:
                        print(
                            "Iteration {} (epoch {}, batch {}/{})".format(
                                self.iter_steps + 1, epoch + 1, bi + 1, num_blocks
                            ),
                            end="",
                        )
                    if callbacks is not None:
                        for cb in callbacks if isinstance(callbacks, (list, tuple)) else (callbacks,):
                            cb(X, self, self.iter_steps)
                    if self.verbose:
                        print()
                    self.iter_steps += 1
        except (KeyboardInterrupt, StopIteration):
            pass
        self.check_errors_()
        return self

    def check_errors_(self):
        """Raises deferred device-side failures (overridden by the models)."""

    @abstractmethod
    def data_log_likelihood_no_rnm(self, X):
        pass

    @abstractmethod
    def data_log_likelihood(self, X):
        pass

    def data_likelihood(self, X):
        return torch.exp_(self.data_log_likelihood(X))

    @abstractmethod
    def compute_elbo(self, X):
        pass

    @abstractmethod
    def log_pred_density(self, X, Y):
        pass

    def pred_density(self, X, Y):
        return torch.exp_(self.log_pred_density(X, Y))

    def load_state_dict(self, state_dict):
        self.block_size = state_dict["block_size"]
        self.verbose = state_dict["verbose"]
        self.iter_steps = state_dict["iter_steps"]

    def state_dict(self):
        return {"block_size": self.block_size, "verbose": self.verbose, "iter_steps": self.iter_steps}

    def hparam_state_dict(self):
        return {"block_size": self.block_size}

    def save(self, fname, state_dict=None):
        d = self.state_dict()
        d.update(state_dict or {})
        torch.save(d, fname)
