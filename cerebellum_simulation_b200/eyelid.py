"""An eyelid-conditioning session in the shape of the reference's driver.

``EyelidSession`` follows ECManagementDelay
(Eyelid_Sim_CBM_Dev/src/ectrial/ecmanagementdelay.cpp) and its base
ECManagementBase (ecmanagementbase.cpp): numTrials trials of interTrialI
steps, CS from csOn to csOff (phasic rates until csPOff) from trial
csStartTN on, the records of numDataTrials trials from dataStartTN on, and
at the end its writeDataToFile output (the state and the ECTrialsData in one
file, the MF rate tables beside it).  The whole session runs on the device as
one protocol; the three ways the driver gets its MF rate tables are the three
constructors:

* ``EyelidSession(state, mf_population, ...)``: tables given, e.g. from
  ``networks.MFPopulation.random`` (the driver's parameter constructor,
  ecmanagementdelay.cpp:10-24, whose network generation is the reference's
  own and not part of this package);
* ``EyelidSession.resume(session_path, ...)``: the state and MF histogram of
  an earlier session file, the tables re-estimated from that histogram
  (ecmanagementdelay.cpp:26-50);
* ``EyelidSession.from_files(state_path, mf_path, ...)``: a state file and a
  file of tables (ecmanagementdelay.cpp:52-70).
"""
from . import CBMSimCore, CBMState, eyelid_protocol_defaults
from .networks import MFPopulation
from .trialdata import read_session


class EyelidSession:
    def __init__(self, state, mf_population, rand_seed, num_trials, iti, cs_on, cs_off, cs_p_off, cs_start_trial,
                 data_start_trial, num_data_trials, device=0, sim_factory=CBMSimCore, **protocol):
        self.state = state
        self.mf_population = mf_population
        self.rand_seed = int(rand_seed)
        self.num_trials = int(num_trials)
        # ECManagementBase's trial clock (ecmanagementbase.cpp:64-100) and
        # ECManagementDelay::initialize (ecmanagementdelay.cpp:72-170): MF
        # generator seeded with randSeed, the driver's plasticity steps and
        # eyelid integrator, 500 ms either side of the CS
        self.protocol = eyelid_protocol_defaults(
            state, trialSteps=int(iti), csOn=int(cs_on), csOff=int(cs_off), csPhasicOff=int(cs_p_off),
            csStartTrial=int(cs_start_trial), dataStartTrial=int(data_start_trial),
            numDataTrials=int(num_data_trials), mfSeed=self.rand_seed, **protocol)
        self.device = device
        self._sim_factory = sim_factory
        self.sim = None

    @classmethod
    def resume(cls, session_path, rand_seed, num_trials, iti, cs_on, cs_off, cs_p_off, cs_start_trial,
               data_start_trial, num_data_trials, **kw):
        state, data = read_session(session_path)
        h = data["header"]
        # ECMFPopulation(ECTrialsData *) takes the bin width and trial count of the file's "mf" histogram
        pop = MFPopulation.from_trial_data(data["psh"]["mf"], data["psh_trials"]["mf"],
                                           data["psh_bin_steps"]["mf"], h["msPreCS"], h["msCS"])
        return cls(state, pop, rand_seed, num_trials, iti, cs_on, cs_off, cs_p_off, cs_start_trial,
                   data_start_trial, num_data_trials, **kw)

    @classmethod
    def from_files(cls, state_path, mf_path, rand_seed, num_trials, iti, cs_on, cs_off, cs_p_off, cs_start_trial,
                   data_start_trial, num_data_trials, **kw):
        return cls(CBMState(state_path), MFPopulation.read(mf_path), rand_seed, num_trials, iti, cs_on, cs_off,
                   cs_p_off, cs_start_trial, data_start_trial, num_data_trials, **kw)

    def run(self, chunk=250):
        """All trials on the device, recording the driver's ECTrialsData;
        the NC->IO draws are keyed by randSeed, as the driver's CBMSimCore
        is built (ecmanagementbase.cpp:42)."""
        self.sim = self._sim_factory(self.state, [self.rand_seed], device=self.device)
        self.sim.set_eyelid_protocol(self.mf_population.rates(), **self.protocol)
        self.sim.record_gr()
        self.sim.record_trial_data()
        self.sim.run(self.num_trials * self.protocol["trialSteps"], chunk=chunk)
        return self.sim

    def write_data_to_file(self, path):
        """ECManagementDelay::writeDataToFile (ecmanagementdelay.cpp:275-290)."""
        if self.sim is None:
            raise RuntimeError("run the session first")
        self.sim.write_session(path, self.mf_population)
